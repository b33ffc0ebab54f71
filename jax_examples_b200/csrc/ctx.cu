// Host side of libjqc.so: context, basis upload, shell-pair build with
// Schwarz bounds, class-sorted work lists and the extern "C" entry points.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "kernels.cuh"

namespace jqc {

// ------------------------------------------------------------------ errors
static thread_local std::string g_last_error;
void set_error(const std::string& msg) { g_last_error = msg; }

#define JQC_REQUIRE(cond, code, msg) \
  do {                               \
    if (!(cond)) {                   \
      set_error(msg);                \
      return code;                   \
    }                                \
  } while (0)

struct OneEParams {
  int n_shell, n, n_atom;
  const int* l;
  const int* nprim;
  const int* prim_off;
  const double* exps;
  const double* coefs;
  const double* centres;
  const int* ao;
  const double* atom_xyz;
  const double* atom_Z;
  const int* shell_mol;  // molecule of each shell / atom (nullptr: one molecule)
  const int* atom_mol;
  const double* boys;
  double* S;
  double* T;
  double* V;
};
cudaError_t launch_one_e(const OneEParams& p, cudaStream_t s);

cudaError_t fma_peak(bool fp32, int blocks, int iters, void* sink, cudaStream_t s, float* ms);
cudaError_t launch_jk64_lo(int qc, const JKParams& p, cudaStream_t s);
cudaError_t launch_jk64_hi(int qc, const JKParams& p, cudaStream_t s);
cudaError_t launch_jk32_lo(int qc, const JKParams& p, cudaStream_t s);
cudaError_t launch_jk32_hi(int qc, const JKParams& p, cudaStream_t s);
cudaError_t launch_jk(int qc, bool fp32, const JKParams& p, cudaStream_t s) {
  if (p.engine == kEngineCol) return launch_col_jk(qc, fp32, p, s);
  if (p.engine == kEngineWarp || !is_reg_class(qc)) {
    const int pb = qc_bra(qc), pk = qc_ket(qc);
    return launch_warp_jk(pc_la(pb), pc_lb(pb), pc_la(pk), pc_lb(pk), fp32, p, s);
  }
  if (qc < 10) return fp32 ? launch_jk32_lo(qc, p, s) : launch_jk64_lo(qc, p, s);
  return fp32 ? launch_jk32_hi(qc, p, s) : launch_jk64_hi(qc, p, s);
}

// ---------------------------------------------------------- device buffer
template <typename T>
struct DevBuf {
  T* ptr = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    n = 0;
  }
  cudaError_t reserve(size_t count) {
    if (count <= n && ptr) return cudaSuccess;
    release();
    if (count == 0) return cudaSuccess;
    cudaError_t e = cudaMalloc(&ptr, count * sizeof(T));
    if (e == cudaSuccess) n = count;
    return e;
  }
  cudaError_t upload(const std::vector<T>& h, cudaStream_t s) {
    cudaError_t e = reserve(h.size());
    if (e != cudaSuccess || h.empty()) return e;
    return cudaMemcpyAsync(ptr, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, s);
  }
};

// ------------------------------------------------------------ Boys tables
void boys_fill_table(double* tab) {
  // F_m(T_i) by the convergent series e^{-T} sum_k (2T)^k / ((2m+1)(2m+3)...(2m+2k+1))
  // at the top order, then downward recursion, all in long double.
  const int top = kBoysCols - 1;
  for (int i = 0; i < kBoysRows; ++i) {
    const long double t = (long double)i / kBoysGridInv;
    long double term = 1.0L / (2 * top + 1), sum = term;
    for (int k = 1; k < 2000; ++k) {
      term *= 2.0L * t / (2 * top + 2 * k + 1);
      sum += term;
      if (term < sum * 1e-22L) break;
    }
    long double e = expl(-t);
    long double f = e * sum;
    tab[i * kBoysCols + top] = (double)f;
    for (int m = top - 1; m >= 0; --m) {
      f = (2.0L * t * f + e) / (2 * m + 1);
      tab[i * kBoysCols + m] = (double)f;
    }
  }
}

int boys_tables_all(int device, BoysTables* out) {
  static std::mutex mu;
  static std::vector<BoysTables> tabs;
  std::lock_guard<std::mutex> lock(mu);
  int ndev = 0;
  JQC_CUDA_CHECK(cudaGetDeviceCount(&ndev));
  JQC_REQUIRE(device >= 0 && device < ndev, JQC_ERR_INVALID, "invalid CUDA device");
  if ((int)tabs.size() < ndev) tabs.resize(ndev, BoysTables{nullptr, nullptr, nullptr, nullptr});
  if (!tabs[device].t64) {
    std::vector<double> h(kBoysRows * kBoysCols);
    boys_fill_table(h.data());
    std::vector<float> hf(h.begin(), h.end());
    std::vector<double> ha(kBoysAlignedSize);
    for (int M = 0; M <= kBoysMaxM; ++M)
      for (int i = 0; i < kBoysRows; ++i)
        for (int k = 0; k < kBoysARow; ++k)
          ha[((size_t)M * kBoysRows + i) * kBoysARow + k] = h[(size_t)i * kBoysCols + M + k] * inv_factorial(k);
    for (int i = 0; i < kBoysExpRows; ++i) ha[kBoysExpOff + i] = (double)expl(-(long double)i / kBoysGridInv);
    std::vector<float> haf(ha.begin(), ha.end());
    int prev = 0;
    JQC_CUDA_CHECK(cudaGetDevice(&prev));
    JQC_CUDA_CHECK(cudaSetDevice(device));
    double *p64 = nullptr, *a64 = nullptr;
    float *p32 = nullptr, *a32 = nullptr;
    JQC_CUDA_CHECK(cudaMalloc(&p64, h.size() * sizeof(double)));
    JQC_CUDA_CHECK(cudaMalloc(&p32, hf.size() * sizeof(float)));
    JQC_CUDA_CHECK(cudaMalloc(&a64, ha.size() * sizeof(double)));
    JQC_CUDA_CHECK(cudaMalloc(&a32, haf.size() * sizeof(float)));
    JQC_CUDA_CHECK(cudaMemcpy(p64, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice));
    JQC_CUDA_CHECK(cudaMemcpy(p32, hf.data(), hf.size() * sizeof(float), cudaMemcpyHostToDevice));
    JQC_CUDA_CHECK(cudaMemcpy(a64, ha.data(), ha.size() * sizeof(double), cudaMemcpyHostToDevice));
    JQC_CUDA_CHECK(cudaMemcpy(a32, haf.data(), haf.size() * sizeof(float), cudaMemcpyHostToDevice));
    JQC_CUDA_CHECK(cudaSetDevice(prev));
    tabs[device] = BoysTables{p64, p32, a64, a32};
  }
  *out = tabs[device];
  return JQC_OK;
}

int boys_tables(int device, const double** d64, const float** d32) {
  BoysTables t;
  int rc = boys_tables_all(device, &t);
  if (rc) return rc;
  *d64 = t.t64;
  *d32 = t.t32;
  return JQC_OK;
}

// ---------------------------------------------------------------- tasks
struct TaskSet {
  bool valid = false;
  int mode = -1;
  double mixed_tau = -1.0;
  bool full = false;  // no quartet screening (dense tensor)
  std::vector<Task> h;
  DevBuf<Task> d;
  int off[2][kNumQuartetClasses] = {};
  int cnt[2][kNumQuartetClasses] = {};
  // packed warp groups of the ket-outer register classes (JKParams::groups):
  // gcnt groups, gcnt + 1 boundaries from goff, relative to the list's start
  std::vector<int> gh;
  DevBuf<int> gd;
  int goff[2][kNumQuartetClasses] = {};
  int gcnt[2][kNumQuartetClasses] = {};
  long long n_quartets[2] = {0, 0};
  long long n_prim_quartets = 0;
  long long class_quartets[2][kNumQuartetClasses] = {};
  long long class_prims[2][kNumQuartetClasses] = {};
  // device-side compaction of the lists (inactive molecules of a batch,
  // density screening): one segment per non-empty list, the surviving item
  // indices of segment k at d_items + comp_item_off[k]
  bool comp_ready = false;
  int comp_nseg = 0;
  long long comp_total = 0;
  int comp_seg_of[2][kNumQuartetClasses] = {};  // segment of a list, -1 none
  long long comp_item_off[2 * kNumQuartetClasses] = {};
  DevBuf<int> d_items;
  DevBuf<int> d_counts;
  DevBuf<CompactSeg> d_segs;
  DevBuf<long long> d_seg_start;
  DevBuf<float> d_item_q;  // per item bound of the density test, segment by segment
};

// Pairs of one (class, primitive-pair count, molecule), Q descending.
struct Block {
  int pc, ka, kb, start, count, mol;
};

// Upper bound on primitive quartets one lane evaluates per task (default).
constexpr int kMaxLanePrims = 256;
constexpr int kTuneInts = 4;  // threads, lane_prims, persistent, engine

// Launch shape of one quartet class, picked by the autotuner: threads per
// block, the bra primitive-pair chunk (at most lane_prims primitive quartets
// per lane and task) and whether the grid is capped at the resident blocks.
struct ClassTune {
  int threads = 128;
  int lane_prims = kMaxLanePrims;
  int persistent = 0;
  int engine = -1;  // JKEngine; -1: the class's default
};

// Default engine of a class: the register kernels where they exist, else the
// column engine, else the runtime-class warp engine.
static int default_engine(int qc) {
  if (qc == 19 || qc == 20) return has_col_class(qc) ? kEngineCol : kEngineWarp;
  return is_reg_class(qc) ? kEngineReg : (has_col_class(qc) ? kEngineCol : kEngineWarp);
}
static int class_engine(const ClassTune& t, int qc) { return t.engine < 0 ? default_engine(qc) : t.engine; }

// Gradient: the row engine for the d-bra classes at L >= 5, the register
// kernels up to L = 4, the warp engine otherwise.
static int default_grad_engine(int qc) {
  if (has_grad_row_class(qc) && qc_L(qc) >= 5) return kEngineCol;
  // dp bras in the register kernels: the split sides halve the time
  // ((dp|ss) 4.0 -> 2.2 ms, (dp|ps) 7.4 -> 3.7 ms on (H2O)16); for the other
  // classes computing R twice costs more than the spills it removes
  if (is_grad_reg_class(qc) && qc_bra(qc) == 4) return kGradEngineRegSplit;
  return is_grad_reg_class(qc) ? kEngineReg : kEngineWarp;
}
// The register gradient kernels (one or two sides): 32 kets per task.
static bool grad_reg_engine(int e) { return e == kEngineReg || e == kGradEngineRegSplit; }
static bool grad_engine_valid(int e, int qc) {
  return ((e == kEngineReg || e == kGradEngineRegSplit) && is_grad_reg_class(qc)) ||
         (e == kEngineCol && has_grad_row_class(qc)) || e == kEngineWarp;
}
static bool engine_valid(int e, int qc) {
  return (e == kEngineReg && is_reg_class(qc)) || (e == kEngineCol && has_col_class(qc)) || e == kEngineWarp;
}
constexpr int kNumStreams = 4;

}  // namespace jqc

using namespace jqc;

struct jqc_ctx {
  int device = 0;
  // basis
  int n_shell = 0, n_bf = 0, n_atom = 0;
  std::vector<int> l, nprim, prim_off, ao, atom;
  std::vector<double> exps, coefs, centres, atom_xyz, atom_Z;
  DevBuf<double> d_centres;
  DevBuf<int> d_ao, d_l, d_atom, d_nprim, d_prim_off;
  DevBuf<double> d_atom_xyz, d_atom_Z, d_exps, d_coefs;
  bool basis_ready = false;
  // batch partition: molecule of each shell / atom (one molecule by default)
  int n_mol = 1;
  std::vector<int> shell_mol, atom_mol;
  std::vector<int> mol_active;  // empty: every molecule takes part in the pair list
  const int* d_mol_active = nullptr;  // caller's device flags read by every J/K build (nullptr: off)
  DevBuf<int> d_shell_mol, d_atom_mol;
  // pairs (sorted: block by (class, K_a, K_b), Q descending inside)
  bool pairs_ready = false;
  double tau = 0.0;
  long long n_pairs_all = 0;
  std::vector<ShellPair> pairs;
  std::vector<Block> blocks;
  std::vector<double> Qmat;  // n_shell x n_shell, original order
  DevBuf<ShellPair> d_pairs;
  DevBuf<PrimPair> d_pp;
  DevBuf<PrimPairF> d_ppf;
  // work lists: one per (precision mode, mixed_tau) in use, plus the dense one
  std::vector<TaskSet*> jk_cache;
  TaskSet* jk_cur = nullptr;
  TaskSet full_tasks;
  TaskSet grad_tasks;  // one screened quartet per task, whole contractions
  // scratch
  DevBuf<float> d_dmax;
  DevBuf<double> d_pair_force;  // gradient: 6 force components per kept shell pair
  cudaStream_t side[kNumStreams] = {};
  cudaEvent_t ev_fork = nullptr, ev_join[kNumStreams] = {};
  cudaEvent_t ev_t0 = nullptr, ev_t1 = nullptr;  // per-class timing
  const double* boys64 = nullptr;
  const float* boys32 = nullptr;
  const double* boysA64 = nullptr;  // aligned per-order tables (hot kernels)
  const float* boysA32 = nullptr;
  double prim_tau = 0.0;
  ClassTune tune[kNumQuartetClasses];
  int grad_engine[kNumQuartetClasses];  // JKEngine numbering: 0 register, 1 row engine, 2 warp
  // CUDA graphs captured through jqc_graph_begin / jqc_graph_end
  std::vector<cudaGraphExec_t> graphs;
};

namespace jqc {

// Primitive pairs of shell pair (a, b).  A pair whose magnitude
// |K_AB c_a c_b| pi^{5/4} p^{-5/4} (the s-type sqrt((ab|ab)) of the
// primitive pair) is below prim_tau contributes nothing at that level to any
// integral and is dropped.
static void make_prim_pairs(const jqc_ctx* c, int a, int b, std::vector<PrimPair>& out) {
  const double* A = &c->centres[3 * a];
  const double* B = &c->centres[3 * b];
  const double dx = A[0] - B[0], dy = A[1] - B[1], dz = A[2] - B[2];
  const double ab2 = dx * dx + dy * dy + dz * dz;
  for (int i = 0; i < c->nprim[a]; ++i)
    for (int j = 0; j < c->nprim[b]; ++j) {
      const double al = c->exps[c->prim_off[a] + i], be = c->exps[c->prim_off[b] + j];
      const double p = al + be;
      PrimPair q;
      q.p = p;
      q.Px = (al * A[0] + be * B[0]) / p;
      q.Py = (al * A[1] + be * B[1]) / p;
      q.Pz = (al * A[2] + be * B[2]) / p;
      q.K = std::exp(-(al * be / p) * ab2) * c->coefs[c->prim_off[a] + i] * c->coefs[c->prim_off[b] + j];
      q.alpha = al;
      q.beta = be;
      q.h = 0.5 / p;
      const double mag = std::fabs(q.K) * 4.1606878161 * std::pow(p, -1.25);  // pi^{5/4}
      if (c->prim_tau > 0.0 && mag < c->prim_tau) continue;
      out.push_back(q);
    }
}

// Number of leading entries k in [0, limit) of a Q-descending block with
// Qi * Q[k] >= thr.
static int prefix_count(const std::vector<ShellPair>& pairs, int start, int limit, double Qi, double thr) {
  if (thr <= 0.0) return limit;
  int lo = 0, hi = limit;
  while (lo < hi) {
    int mid = (lo + hi) / 2;
    if (Qi * pairs[start + mid].Q >= thr)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

// Tasks and counters of the bra pairs [g0, g1) (one worker of build_tasks).
struct TaskPart {
  std::vector<Task> lists[2][kNumQuartetClasses];
  long long nq[2] = {0, 0}, npq = 0;
  long long cq[2][kNumQuartetClasses] = {}, cp[2][kNumQuartetClasses] = {};
};

static void build_task_part(const jqc_ctx* c, TaskPart& out, int g0, int g1, const std::vector<int>& block_of,
                            const std::vector<std::vector<int>>& mol_blocks, int mode, double mixed_tau, bool full,
                            bool grad) {
  const double tau = full ? 0.0 : c->tau;
  for (int gi = g0; gi < g1; ++gi) {
    const size_t cb = (size_t)block_of[gi];
    const Block& B = c->blocks[cb];
    const int pi = gi - B.start;
    const double Qi = c->pairs[gi].Q;
    for (const int ckb : mol_blocks[B.mol]) {
      const size_t ck = (size_t)ckb;
      if (ck > cb) break;
      const Block& K = c->blocks[ck];
      const int limit = (ck == cb) ? pi + 1 : K.count;
      const int n_all = prefix_count(c->pairs, K.start, limit, Qi, tau);
      int n64 = n_all;
      if (mode == JQC_PREC_FP32) n64 = 0;
      if (mode == JQC_PREC_MIXED) n64 = std::min(n_all, prefix_count(c->pairs, K.start, limit, Qi, mixed_tau));
      const int qc = quartet_class(B.pc, K.pc);
      const int seg[3] = {0, n64, n_all};
      // Split the bra primitive pairs so one lane does at most ~lane_prims
      // primitive quartets per task (the tensor keeps whole quartets).
      const int nbp = c->pairs[gi].npp, nkp = K.ka * K.kb;
      int chunk = nbp;
      if (!full) chunk = std::max(1, std::min(nbp, c->tune[qc].lane_prims / std::max(1, nkp)));
      // Register kernels: up to 32 kets per warp task (one per lane); the
      // other engines: one ket per task, so every quartet gets its own warp.
      const int per_task =
          grad ? (grad_reg_engine(c->grad_engine[qc]) ? 32 : 1) : (class_engine(c->tune[qc], qc) == kEngineReg ? 32 : 1);
      for (int prec = 0; prec < 2; ++prec) {
        for (int k0 = seg[prec]; k0 < seg[prec + 1]; k0 += per_task) {
          for (int b0 = 0; b0 < nbp; b0 += chunk) {
            Task t;
            t.bra = gi;
            t.ket0 = K.start + k0;
            t.nket = std::min(per_task, seg[prec + 1] - k0);
            t.flags = b0 | (std::min(nbp, b0 + chunk) << 16);
            out.lists[prec][qc].push_back(t);
          }
        }
        out.nq[prec] += seg[prec + 1] - seg[prec];
        out.cq[prec][qc] += seg[prec + 1] - seg[prec];
        out.cp[prec][qc] += (long long)(seg[prec + 1] - seg[prec]) * nbp * nkp;
      }
      out.npq += (long long)n_all * c->pairs[gi].npp * K.ka * K.kb;
    }
  }
}

// Angular momentum sum of the bra pair of quartet class qc.
static int qc_bra_lsum(int qc) { return pc_la(qc_bra(qc)) + pc_lb(qc_bra(qc)); }

// Packs the tasks h[base, base + n) (one class list, sorted by descending
// lane cost) into warp groups of at most 32 kets: inside each run of equal
// cost, full tasks stay alone and the partial ones are paired largest with
// smallest; the tasks of a group are made contiguous.  Appends the group
// boundaries (relative to base, n_groups + 1 of them) to g and returns the
// number of groups.
template <typename Cost>
static int pack_groups(std::vector<Task>& h, size_t base, size_t n, std::vector<int>& g, Cost lane_cost) {
  std::vector<Task> part, out;
  out.reserve(n);
  int groups = 0;
  g.push_back(0);
  size_t i0 = 0;
  while (i0 < n) {
    size_t i1 = i0;
    while (i1 < n && lane_cost(h[base + i1]) == lane_cost(h[base + i0])) ++i1;
    part.clear();
    for (size_t k = i0; k < i1; ++k) {
      const Task& t = h[base + k];
      if (t.nket >= 32) {
        out.push_back(t);
        g.push_back((int)out.size());
        ++groups;
      } else {
        part.push_back(t);
      }
    }
    std::stable_sort(part.begin(), part.end(), [](const Task& a, const Task& b) { return a.nket > b.nket; });
    size_t lo = 0, hi = part.size();
    while (lo < hi) {
      int fill = part[lo].nket;
      out.push_back(part[lo++]);
      while (lo < hi && fill + part[hi - 1].nket <= 32) {
        fill += part[hi - 1].nket;
        out.push_back(part[--hi]);
      }
      g.push_back((int)out.size());
      ++groups;
    }
    i0 = i1;
  }
  std::copy(out.begin(), out.end(), h.begin() + (long)base);
  return groups;
}

static int build_tasks(jqc_ctx* c, TaskSet& ts, int mode, double mixed_tau, bool full, cudaStream_t s,
                       bool grad = false) {
  // Quartets pair a bra and a ket of the same molecule: ket blocks by molecule.
  std::vector<std::vector<int>> mol_blocks(c->n_mol);
  for (size_t cb = 0; cb < c->blocks.size(); ++cb) mol_blocks[c->blocks[cb].mol].push_back((int)cb);
  const int n_pairs = (int)c->pairs.size();
  std::vector<int> block_of(n_pairs);
  for (size_t cb = 0; cb < c->blocks.size(); ++cb)
    for (int k = 0; k < c->blocks[cb].count; ++k) block_of[c->blocks[cb].start + k] = (int)cb;
  // Bra pairs split over host threads; the parts are concatenated in order,
  // so the work list does not depend on the thread count.
  int nthreads = (int)std::min<unsigned>(16u, std::max(1u, std::thread::hardware_concurrency()));
  if (n_pairs < 4096) nthreads = 1;
  std::vector<TaskPart> parts(nthreads);
  {
    std::vector<std::thread> pool;
    for (int t = 0; t < nthreads; ++t) {
      const int g0 = (int)((long long)n_pairs * t / nthreads), g1 = (int)((long long)n_pairs * (t + 1) / nthreads);
      if (nthreads == 1)
        build_task_part(c, parts[t], g0, g1, block_of, mol_blocks, mode, mixed_tau, full, grad);
      else
        pool.emplace_back(build_task_part, c, std::ref(parts[t]), g0, g1, std::cref(block_of), std::cref(mol_blocks),
                          mode, mixed_tau, full, grad);
    }
    for (auto& th : pool) th.join();
  }
  long long nq[2] = {0, 0}, npq = 0;
  long long cq[2][kNumQuartetClasses] = {}, cp[2][kNumQuartetClasses] = {};
  for (const TaskPart& p : parts) {
    nq[0] += p.nq[0];
    nq[1] += p.nq[1];
    npq += p.npq;
    for (int prec = 0; prec < 2; ++prec)
      for (int qc = 0; qc < kNumQuartetClasses; ++qc) {
        cq[prec][qc] += p.cq[prec][qc];
        cp[prec][qc] += p.cp[prec][qc];
      }
  }
  // Every (precision path, class) list is finished on its own, the lists in
  // parallel: the parts are concatenated in bra order, the tasks ordered
  // longest first (cost = lane primitive quartets = bra primitive chunk x
  // ket primitive pairs; a stable counting sort, linear in the number of
  // tasks), and the ket-outer register classes packed into warp groups.
  constexpr int kSegs = 2 * kNumQuartetClasses;
  std::vector<std::vector<Task>> seg_tasks(kSegs);
  std::vector<std::vector<int>> seg_groups(kSegs);
  std::vector<int> seg_ngroups(kSegs, 0);
  auto finish_segment = [&](int sg) {
    const int prec = sg / kNumQuartetClasses, qc = sg % kNumQuartetClasses;
    size_t total = 0;
    for (const TaskPart& p : parts) total += p.lists[prec][qc].size();
    std::vector<int> cost(total), count;
    int cmax = 0;
    {
      size_t k = 0;
      for (const TaskPart& p : parts)
        for (const Task& t : p.lists[prec][qc]) {
          cost[k] = ((t.flags >> 16) - (t.flags & 0xffff)) * c->pairs[t.ket0].npp;
          cmax = std::max(cmax, cost[k]);
          ++k;
        }
    }
    count.assign(cmax + 2, 0);
    for (size_t k = 0; k < total; ++k) ++count[cmax - cost[k] + 1];  // descending cost
    for (int b = 1; b <= cmax + 1; ++b) count[b] += count[b - 1];
    std::vector<Task>& out = seg_tasks[sg];
    out.resize(total);
    {
      size_t k = 0;
      for (const TaskPart& p : parts)
        for (const Task& t : p.lists[prec][qc]) out[count[cmax - cost[k++]]++] = t;
    }
    if (!full && !grad && qc_bra_lsum(qc) <= kKetOuterMaxLab && class_engine(c->tune[qc], qc) == kEngineReg)
      seg_ngroups[sg] = pack_groups(out, 0, total, seg_groups[sg], [c](const Task& t) {
        return ((t.flags >> 16) - (t.flags & 0xffff)) * c->pairs[t.ket0].npp;
      });
  };
  {
    std::vector<std::thread> pool;
    std::atomic<int> next{0};
    const int nw = std::max(1, std::min(nthreads, kSegs));
    for (int w = 0; w < nw; ++w)
      pool.emplace_back([&]() {
        for (int sg = next++; sg < kSegs; sg = next++) finish_segment(sg);
      });
    for (auto& th : pool) th.join();
  }
  parts.clear();
  ts.h.clear();
  ts.gh.clear();
  size_t total_tasks = 0, total_groups = 0;
  for (int sg = 0; sg < kSegs; ++sg) {
    total_tasks += seg_tasks[sg].size();
    total_groups += seg_groups[sg].size();
  }
  ts.h.resize(total_tasks);
  ts.gh.reserve(total_groups);
  size_t base = 0;
  for (int sg = 0; sg < kSegs; ++sg) {
    const int prec = sg / kNumQuartetClasses, qc = sg % kNumQuartetClasses;
    ts.off[prec][qc] = (int)base;
    ts.cnt[prec][qc] = (int)seg_tasks[sg].size();
    std::copy(seg_tasks[sg].begin(), seg_tasks[sg].end(), ts.h.begin() + (long)base);
    base += seg_tasks[sg].size();
    ts.goff[prec][qc] = (int)ts.gh.size();
    ts.gcnt[prec][qc] = seg_ngroups[sg];
    ts.gh.insert(ts.gh.end(), seg_groups[sg].begin(), seg_groups[sg].end());
    std::vector<Task>().swap(seg_tasks[sg]);
  }
  JQC_CUDA_CHECK(ts.d.upload(ts.h, s));
  JQC_CUDA_CHECK(ts.gd.upload(ts.gh, s));
  ts.n_quartets[0] = nq[0];
  ts.n_quartets[1] = nq[1];
  ts.n_prim_quartets = npq;
  std::memcpy(ts.class_quartets, cq, sizeof(cq));
  std::memcpy(ts.class_prims, cp, sizeof(cp));
  ts.mode = mode;
  ts.mixed_tau = mixed_tau;
  ts.full = full;
  ts.valid = true;
  // Segments for the device-side compaction of the lists (used while
  // jqc_set_molecule_activity is set and by density-screened builds), with
  // each item's largest float(Q_bra) float(Q_ket): the kernels' density bound
  // is that times 2 max|D block|, computed with the same operations.
  ts.comp_ready = false;
  if (!full && !grad) {
    std::vector<CompactSeg> segs;
    std::vector<long long> starts;
    std::vector<float> item_q;
    long long tot = 0;
    int nseg = 0;
    for (int prec = 0; prec < 2; ++prec)
      for (int qc = 0; qc < kNumQuartetClasses; ++qc) {
        ts.comp_seg_of[prec][qc] = -1;
        const int items = ts.gcnt[prec][qc] > 0 ? ts.gcnt[prec][qc] : ts.cnt[prec][qc];
        if (ts.cnt[prec][qc] == 0) continue;
        ts.comp_seg_of[prec][qc] = nseg;
        ts.comp_item_off[nseg] = tot;
        starts.push_back(tot);
        segs.push_back(CompactSeg{nullptr, nullptr, items, nullptr, nullptr, nullptr});
        const Task* lt = ts.h.data() + ts.off[prec][qc];
        auto task_q = [&](const Task& t) {
          return float(c->pairs[t.bra].Q) * float(c->pairs[t.ket0].Q);  // ket runs: Q-descending
        };
        for (int it = 0; it < items; ++it) {
          float q = 0.f;
          if (ts.gcnt[prec][qc] > 0) {
            const int* gb = ts.gh.data() + ts.goff[prec][qc];
            for (int t = gb[it]; t < gb[it + 1]; ++t) q = std::max(q, task_q(lt[t]));
          } else {
            q = task_q(lt[it]);
          }
          item_q.push_back(q);
        }
        tot += items;
        ++nseg;
      }
    starts.push_back(tot);
    JQC_CUDA_CHECK(ts.d_items.reserve((size_t)std::max<long long>(tot, 1)));
    JQC_CUDA_CHECK(ts.d_counts.reserve((size_t)std::max(nseg, 1)));
    if (item_q.empty()) item_q.push_back(0.f);
    JQC_CUDA_CHECK(ts.d_item_q.upload(item_q, s));
    int k = 0;
    for (int prec = 0; prec < 2; ++prec)
      for (int qc = 0; qc < kNumQuartetClasses; ++qc) {
        if (ts.comp_seg_of[prec][qc] < 0) continue;
        CompactSeg& sg = segs[k];
        sg.tasks = ts.d.ptr + ts.off[prec][qc];
        sg.groups = ts.gcnt[prec][qc] > 0 ? ts.gd.ptr + ts.goff[prec][qc] : nullptr;
        sg.out = ts.d_items.ptr + ts.comp_item_off[k];
        sg.count = ts.d_counts.ptr + k;
        sg.item_q = ts.d_item_q.ptr + ts.comp_item_off[k];
        ++k;
      }
    JQC_CUDA_CHECK(ts.d_segs.upload(segs, s));
    JQC_CUDA_CHECK(ts.d_seg_start.upload(starts, s));
    JQC_CUDA_CHECK(cudaStreamSynchronize(s));
    ts.comp_nseg = nseg;
    ts.comp_total = tot;
    ts.comp_ready = true;
  }
  return JQC_OK;
}

static int ensure_tasks(jqc_ctx* c, TaskSet& ts, int mode, double mixed_tau, bool full, cudaStream_t s) {
  if (mode != JQC_PREC_MIXED) mixed_tau = 0.0;
  if (ts.valid && ts.mode == mode && ts.mixed_tau == mixed_tau && ts.full == full) return JQC_OK;
  return build_tasks(c, ts, mode, mixed_tau, full, s);
}

static void drop_graphs(jqc_ctx* c);

// J/K work list for (mode, mixed_tau), built once and kept (a few per context).
static int ensure_jk_tasks(jqc_ctx* c, int mode, double mixed_tau, cudaStream_t s) {
  if (mode != JQC_PREC_MIXED) mixed_tau = 0.0;
  for (TaskSet* ts : c->jk_cache)
    if (ts->valid && ts->mode == mode && ts->mixed_tau == mixed_tau) {
      c->jk_cur = ts;
      return JQC_OK;
    }
  if (c->jk_cache.size() >= 4) {
    drop_graphs(c);
    delete c->jk_cache.front();
    c->jk_cache.erase(c->jk_cache.begin());
  }
  TaskSet* ts = new TaskSet();
  int rc = build_tasks(c, *ts, mode, mixed_tau, false, s);
  if (rc) {
    delete ts;
    return rc;
  }
  c->jk_cache.push_back(ts);
  c->jk_cur = ts;
  return JQC_OK;
}

// Captured graphs hold pointers to the work lists and pair data: whatever
// frees or replaces those destroys the graphs first (their ids then fail).
static void drop_graphs(jqc_ctx* c) {
  for (cudaGraphExec_t& g : c->graphs)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
}

static void drop_jk_tasks(jqc_ctx* c) {
  drop_graphs(c);
  for (TaskSet* ts : c->jk_cache) delete ts;
  c->jk_cache.clear();
  c->jk_cur = nullptr;
}

static int select_device(const jqc_ctx* c) {
  JQC_CUDA_CHECK(cudaSetDevice(c->device));
  return JQC_OK;
}

static bool stream_capturing(cudaStream_t s) {
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &st) != cudaSuccess) return false;
  return st == cudaStreamCaptureStatusActive;
}

static TaskSet* find_jk_tasks(jqc_ctx* c, int mode, double mixed_tau) {
  if (mode != JQC_PREC_MIXED) mixed_tau = 0.0;
  for (TaskSet* ts : c->jk_cache)
    if (ts->valid && ts->mode == mode && ts->mixed_tau == mixed_tau) return ts;
  return nullptr;
}

// One J/K build over work list `ts`: zero J/K, density maxima (when dmax is
// given), the class kernels on the side streams (forked from and joined back
// into s; they only add into J/K with atomics), then J = A + A^T, K = B + B^T.
// With class_ms the classes run one after another on s, each timed.  Only
// stream operations: no allocation, no host synchronisation except for the
// timed form, so the untimed form can be captured into a CUDA graph.
static int run_jk_set(jqc_ctx* c, const TaskSet* ts, int n_dens, const double* D, double* J, double* K,
                      float* dmax, float* dmax_top, double dens_tau, cudaStream_t s, double* class_ms) {
  const int n = c->n_bf;
  const size_t nn = (size_t)n * n * n_dens;
  JQC_CUDA_CHECK(cudaMemsetAsync(J, 0, nn * sizeof(double), s));
  JQC_CUDA_CHECK(cudaMemsetAsync(K, 0, nn * sizeof(double), s));
  if (class_ms)
    for (int k = 0; k < 2 * kNumQuartetClasses; ++k) class_ms[k] = 0.0;
  if (dens_tau > 0.0 && dmax != nullptr) {
    JQC_CUDA_CHECK(launch_dmax(D, n_dens, n, c->n_shell, c->d_ao.ptr, c->d_l.ptr, dmax, dmax_top, s));
  } else {
    dmax = nullptr;
    dmax_top = nullptr;
  }
  // Molecules flagged inactive, and work items whose every lane is below the
  // density bound, leave the build before any class kernel runs: the lists
  // are compacted on the device.
  const bool compact = (c->d_mol_active != nullptr || dmax_top != nullptr) && ts->comp_ready && ts->comp_nseg > 0;
  if (compact) {
    JQC_CUDA_CHECK(cudaMemsetAsync(ts->d_counts.ptr, 0, (size_t)ts->comp_nseg * sizeof(int), s));
    JQC_CUDA_CHECK(launch_compact(ts->d_segs.ptr, ts->d_seg_start.ptr, ts->comp_nseg, ts->comp_total,
                                  c->d_pairs.ptr, c->d_shell_mol.ptr, c->d_mol_active, dmax_top,
                                  (float)dens_tau, s));
  }
  if (!class_ms) {
    JQC_CUDA_CHECK(cudaEventRecord(c->ev_fork, s));
    for (int i = 0; i < kNumStreams; ++i) JQC_CUDA_CHECK(cudaStreamWaitEvent(c->side[i], c->ev_fork, 0));
  }
  int li = 0;
  for (int prec = 0; prec < 2; ++prec)
    for (int qc = 0; qc < kNumQuartetClasses; ++qc) {
      JKParams p;
      p.tasks = ts->d.ptr + ts->off[prec][qc];
      p.n_tasks = ts->cnt[prec][qc];
      if (p.n_tasks == 0) continue;
      p.pairs = c->d_pairs.ptr;
      p.pp = prec ? (const void*)c->d_ppf.ptr : (const void*)c->d_pp.ptr;
      p.centres = c->d_centres.ptr;
      p.ao = c->d_ao.ptr;
      p.boys = prec ? (const void*)c->boys32 : (const void*)c->boys64;
      p.boys_al = prec ? (const void*)c->boysA32 : (const void*)c->boysA64;
      p.D = D;
      p.J = J;
      p.K = K;
      p.n = n;
      p.n_dens = n_dens;
      p.dmax = dmax;
      p.dmax_top = dmax_top;
      p.n_shell = c->n_shell;
      p.dens_tau = (float)dens_tau;
      p.threads = c->tune[qc].threads;
      p.persistent = c->tune[qc].persistent;
      p.engine = class_engine(c->tune[qc], qc);
      if (ts->gcnt[prec][qc] > 0 && p.engine == kEngineReg) {
        p.groups = ts->gd.ptr + ts->goff[prec][qc];
        p.n_groups = ts->gcnt[prec][qc];
      }
      if (compact && ts->comp_seg_of[prec][qc] >= 0) {
        const int sg = ts->comp_seg_of[prec][qc];
        p.items = ts->d_items.ptr + ts->comp_item_off[sg];
        p.n_items = ts->d_counts.ptr + sg;
        if (c->d_mol_active != nullptr) {
          p.shell_mol = c->d_shell_mol.ptr;
          p.mol_active = c->d_mol_active;
        }
      }
      if (class_ms) {
        JQC_CUDA_CHECK(cudaEventRecord(c->ev_t0, s));
        JQC_CUDA_CHECK(launch_jk(qc, prec == 1, p, s));
        JQC_CUDA_CHECK(cudaEventRecord(c->ev_t1, s));
        JQC_CUDA_CHECK(cudaEventSynchronize(c->ev_t1));
        float ms = 0.f;
        JQC_CUDA_CHECK(cudaEventElapsedTime(&ms, c->ev_t0, c->ev_t1));
        class_ms[prec * kNumQuartetClasses + qc] = ms;
      } else {
        JQC_CUDA_CHECK(launch_jk(qc, prec == 1, p, c->side[li++ % kNumStreams]));
      }
    }
  if (!class_ms) {
    for (int i = 0; i < kNumStreams; ++i) {
      JQC_CUDA_CHECK(cudaEventRecord(c->ev_join[i], c->side[i]));
      JQC_CUDA_CHECK(cudaStreamWaitEvent(s, c->ev_join[i], 0));
    }
  }
  JQC_CUDA_CHECK(launch_symmetrize(J, n_dens, n, s));
  JQC_CUDA_CHECK(launch_symmetrize(K, n_dens, n, s));
  return JQC_OK;
}

}  // namespace jqc

// ======================================================================
// extern "C" API
// ======================================================================
extern "C" {

const char* jqc_last_error(void) { return g_last_error.c_str(); }

int jqc_version(void) { return 100; }

int jqc_ctx_create(int device, jqc_ctx** out) {
  JQC_REQUIRE(out != nullptr, JQC_ERR_INVALID, "jqc_ctx_create: out is null");
  int ndev = 0;
  JQC_CUDA_CHECK(cudaGetDeviceCount(&ndev));
  JQC_REQUIRE(device >= 0 && device < ndev, JQC_ERR_INVALID, "jqc_ctx_create: invalid device");
  jqc_ctx* c = new jqc_ctx();
  c->device = device;
  BoysTables bt;
  int rc = boys_tables_all(device, &bt);
  if (rc != JQC_OK) {
    delete c;
    return rc;
  }
  for (int qc = 0; qc < kNumQuartetClasses; ++qc) c->grad_engine[qc] = default_grad_engine(qc);
  c->boys64 = bt.t64;
  c->boys32 = bt.t32;
  c->boysA64 = bt.a64;
  c->boysA32 = bt.a32;
  cudaError_t e = cudaSetDevice(device);
  for (int i = 0; i < kNumStreams && e == cudaSuccess; ++i) {
    e = cudaStreamCreateWithFlags(&c->side[i], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_join[i], cudaEventDisableTiming);
  }
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreate(&c->ev_t0);
  if (e == cudaSuccess) e = cudaEventCreate(&c->ev_t1);
  if (e != cudaSuccess) {
    set_error(std::string("jqc_ctx_create: ") + cudaGetErrorString(e));
    jqc_ctx_destroy(c);
    return JQC_ERR_CUDA;
  }
  *out = c;
  return JQC_OK;
}

int jqc_ctx_destroy(jqc_ctx* ctx) {
  if (ctx) {
    cudaSetDevice(ctx->device);
    for (int i = 0; i < kNumStreams; ++i) {
      if (ctx->side[i]) cudaStreamDestroy(ctx->side[i]);
      if (ctx->ev_join[i]) cudaEventDestroy(ctx->ev_join[i]);
    }
    if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
    if (ctx->ev_t0) cudaEventDestroy(ctx->ev_t0);
    if (ctx->ev_t1) cudaEventDestroy(ctx->ev_t1);
    drop_jk_tasks(ctx);  // destroys the captured graphs too
    delete ctx;
    (void)cudaGetLastError();  // teardown status is not reported to later calls
  }
  return JQC_OK;
}

int jqc_basis_upload(jqc_ctx* c, int n_shell, const int* l, const int* nprim, const int* prim_off, const double* exps,
                     const double* coefs, const double* centres, const int* atom_of_shell, int n_atom,
                     const double* atom_xyz, const double* atom_charge, int cartesian) {
  JQC_REQUIRE(c != nullptr, JQC_ERR_INVALID, "jqc_basis_upload: null context");
  JQC_REQUIRE(n_shell > 0, JQC_ERR_INVALID, "jqc_basis_upload: n_shell must be positive");
  JQC_REQUIRE(cartesian == 1, JQC_ERR_UNSUPPORTED, "jqc_basis_upload: only Cartesian shells are supported");
  JQC_REQUIRE(l && nprim && prim_off && exps && coefs && centres && atom_of_shell, JQC_ERR_INVALID,
              "jqc_basis_upload: null array");
  JQC_REQUIRE(n_atom >= 0 && (n_atom == 0 || (atom_xyz && atom_charge)), JQC_ERR_INVALID,
              "jqc_basis_upload: bad atom arrays");
  int rc = select_device(c);
  if (rc) return rc;
  int np_total = 0;
  for (int s = 0; s < n_shell; ++s) {
    JQC_REQUIRE(l[s] >= 0, JQC_ERR_INVALID, "jqc_basis_upload: negative angular momentum");
    JQC_REQUIRE(l[s] <= kMaxL, JQC_ERR_UNSUPPORTED, "jqc_basis_upload: angular momentum > 2 is not supported");
    JQC_REQUIRE(nprim[s] > 0 && prim_off[s] >= 0, JQC_ERR_INVALID, "jqc_basis_upload: bad primitive range");
    JQC_REQUIRE(atom_of_shell[s] >= 0 && (n_atom == 0 || atom_of_shell[s] < n_atom), JQC_ERR_INVALID,
                "jqc_basis_upload: atom index out of range");
    np_total = std::max(np_total, prim_off[s] + nprim[s]);
  }
  for (int i = 0; i < np_total; ++i) {
    JQC_REQUIRE(std::isfinite(exps[i]) && exps[i] > 0.0, JQC_ERR_INVALID,
                "jqc_basis_upload: exponents must be finite and positive");
    JQC_REQUIRE(std::isfinite(coefs[i]), JQC_ERR_INVALID, "jqc_basis_upload: non-finite coefficient");
  }
  for (int i = 0; i < 3 * n_shell; ++i)
    JQC_REQUIRE(std::isfinite(centres[i]), JQC_ERR_INVALID, "jqc_basis_upload: non-finite centre");
  c->n_shell = n_shell;
  c->l.assign(l, l + n_shell);
  c->nprim.assign(nprim, nprim + n_shell);
  c->prim_off.assign(prim_off, prim_off + n_shell);
  c->exps.assign(exps, exps + np_total);
  c->coefs.assign(coefs, coefs + np_total);
  c->centres.assign(centres, centres + 3 * n_shell);
  c->atom.assign(atom_of_shell, atom_of_shell + n_shell);
  c->n_atom = n_atom;
  c->atom_xyz.assign(atom_xyz ? atom_xyz : centres, atom_xyz ? atom_xyz + 3 * n_atom : centres);
  c->atom_Z.assign(atom_charge ? atom_charge : centres, atom_charge ? atom_charge + n_atom : centres);
  c->ao.resize(n_shell);
  int off = 0;
  for (int s = 0; s < n_shell; ++s) {
    c->ao[s] = off;
    off += ncart(l[s]);
  }
  c->n_bf = off;
  cudaStream_t s0 = 0;
  JQC_CUDA_CHECK(c->d_centres.upload(c->centres, s0));
  JQC_CUDA_CHECK(c->d_ao.upload(c->ao, s0));
  JQC_CUDA_CHECK(c->d_l.upload(c->l, s0));
  JQC_CUDA_CHECK(c->d_atom.upload(c->atom, s0));
  JQC_CUDA_CHECK(c->d_nprim.upload(c->nprim, s0));
  JQC_CUDA_CHECK(c->d_prim_off.upload(c->prim_off, s0));
  JQC_CUDA_CHECK(c->d_exps.upload(c->exps, s0));
  JQC_CUDA_CHECK(c->d_coefs.upload(c->coefs, s0));
  if (n_atom > 0) {
    JQC_CUDA_CHECK(c->d_atom_xyz.upload(c->atom_xyz, s0));
    JQC_CUDA_CHECK(c->d_atom_Z.upload(c->atom_Z, s0));
  }
  c->n_mol = 1;
  c->shell_mol.assign(n_shell, 0);
  c->atom_mol.assign(n_atom, 0);
  c->mol_active.clear();
  JQC_CUDA_CHECK(cudaStreamSynchronize(s0));
  c->basis_ready = true;
  c->pairs_ready = false;
  drop_jk_tasks(c);
  c->full_tasks.valid = false;
  c->grad_tasks.valid = false;
  return JQC_OK;
}

int jqc_batch_partition(jqc_ctx* c, int n_mol, const int* mol_of_atom) {
  JQC_REQUIRE(c != nullptr, JQC_ERR_INVALID, "jqc_batch_partition: null context");
  JQC_REQUIRE(c->basis_ready, JQC_ERR_NOT_READY, "jqc_batch_partition: call jqc_basis_upload first");
  JQC_REQUIRE(c->n_atom > 0, JQC_ERR_NOT_READY, "jqc_batch_partition: the basis was uploaded without atoms");
  JQC_REQUIRE(n_mol >= 1 && n_mol <= c->n_atom, JQC_ERR_INVALID, "jqc_batch_partition: n_mol out of range");
  JQC_REQUIRE(mol_of_atom != nullptr, JQC_ERR_INVALID, "jqc_batch_partition: null mol_of_atom");
  for (int a = 0; a < c->n_atom; ++a)
    JQC_REQUIRE(mol_of_atom[a] >= 0 && mol_of_atom[a] < n_mol, JQC_ERR_INVALID,
                "jqc_batch_partition: molecule index out of range");
  int rc = select_device(c);
  if (rc) return rc;
  c->n_mol = n_mol;
  c->mol_active.clear();
  c->atom_mol.assign(mol_of_atom, mol_of_atom + c->n_atom);
  for (int s = 0; s < c->n_shell; ++s) c->shell_mol[s] = c->atom_mol[c->atom[s]];
  cudaStream_t s0 = 0;
  JQC_CUDA_CHECK(c->d_shell_mol.upload(c->shell_mol, s0));
  JQC_CUDA_CHECK(c->d_atom_mol.upload(c->atom_mol, s0));
  JQC_CUDA_CHECK(cudaStreamSynchronize(s0));
  c->pairs_ready = false;
  drop_jk_tasks(c);
  c->full_tasks.valid = false;
  c->grad_tasks.valid = false;
  return JQC_OK;
}

int jqc_set_geometry(jqc_ctx* c, const double* atom_xyz) {
  JQC_REQUIRE(c != nullptr, JQC_ERR_INVALID, "jqc_set_geometry: null context");
  JQC_REQUIRE(c->basis_ready, JQC_ERR_NOT_READY, "jqc_set_geometry: call jqc_basis_upload first");
  JQC_REQUIRE(c->n_atom > 0, JQC_ERR_NOT_READY, "jqc_set_geometry: the basis was uploaded without atoms");
  JQC_REQUIRE(atom_xyz != nullptr, JQC_ERR_INVALID, "jqc_set_geometry: null atom_xyz");
  for (int i = 0; i < 3 * c->n_atom; ++i)
    JQC_REQUIRE(std::isfinite(atom_xyz[i]), JQC_ERR_INVALID, "jqc_set_geometry: non-finite coordinate");
  int rc = select_device(c);
  if (rc) return rc;
  c->atom_xyz.assign(atom_xyz, atom_xyz + 3 * c->n_atom);
  for (int s = 0; s < c->n_shell; ++s)
    for (int k = 0; k < 3; ++k) c->centres[3 * s + k] = atom_xyz[3 * c->atom[s] + k];
  cudaStream_t s0 = 0;
  JQC_CUDA_CHECK(c->d_centres.upload(c->centres, s0));
  JQC_CUDA_CHECK(c->d_atom_xyz.upload(c->atom_xyz, s0));
  JQC_CUDA_CHECK(cudaStreamSynchronize(s0));
  c->pairs_ready = false;
  drop_jk_tasks(c);
  c->full_tasks.valid = false;
  c->grad_tasks.valid = false;
  return JQC_OK;
}

int jqc_set_molecule_activity(jqc_ctx* c, const int* d_active) {
  JQC_REQUIRE(c != nullptr, JQC_ERR_INVALID, "jqc_set_molecule_activity: null context");
  if (d_active != nullptr) {
    cudaPointerAttributes attr;
    const cudaError_t e = cudaPointerGetAttributes(&attr, d_active);
    (void)cudaGetLastError();
    JQC_REQUIRE(e == cudaSuccess && (attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged),
                JQC_ERR_INVALID, "jqc_set_molecule_activity: the flags must be in device memory");
  }
  if (d_active != c->d_mol_active) drop_graphs(c);  // graphs read the array they were captured with
  c->d_mol_active = d_active;
  return JQC_OK;
}

int jqc_set_molecule_mask(jqc_ctx* c, const int* active) {
  JQC_REQUIRE(c != nullptr, JQC_ERR_INVALID, "jqc_set_molecule_mask: null context");
  JQC_REQUIRE(c->basis_ready, JQC_ERR_NOT_READY, "jqc_set_molecule_mask: call jqc_basis_upload first");
  if (active == nullptr) {
    c->mol_active.clear();
  } else {
    c->mol_active.assign(active, active + c->n_mol);
    for (int& a : c->mol_active) a = a != 0;
  }
  c->pairs_ready = false;
  drop_jk_tasks(c);
  c->full_tasks.valid = false;
  c->grad_tasks.valid = false;
  return JQC_OK;
}

int jqc_pairs_build(jqc_ctx* c, double schwarz_tau, double prim_tau, void* stream) {
  JQC_REQUIRE(c != nullptr, JQC_ERR_INVALID, "jqc_pairs_build: null context");
  JQC_REQUIRE(c->basis_ready, JQC_ERR_NOT_READY, "jqc_pairs_build: call jqc_basis_upload first");
  JQC_REQUIRE(schwarz_tau >= 0.0 && std::isfinite(schwarz_tau), JQC_ERR_INVALID,
              "jqc_pairs_build: schwarz_tau must be >= 0");
  JQC_REQUIRE(prim_tau >= 0.0 && std::isfinite(prim_tau), JQC_ERR_INVALID, "jqc_pairs_build: prim_tau must be >= 0");
  c->prim_tau = prim_tau;
  int rc = select_device(c);
  if (rc) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // 1. all shell pairs a >= b (by l, then index), unsorted
  std::vector<ShellPair> raw;
  std::vector<PrimPair> rawpp;
  std::vector<int> ids[kNumPairClasses];
  for (int i = 0; i < c->n_shell; ++i)
    for (int j = 0; j <= i; ++j) {
      if (c->shell_mol[i] != c->shell_mol[j]) continue;  // no pairs across molecules
      if (!c->mol_active.empty() && !c->mol_active[c->shell_mol[i]]) continue;  // molecule left out
      int a = i, b = j;
      if (c->l[a] < c->l[b]) std::swap(a, b);
      ShellPair sp;
      sp.a = a;
      sp.b = b;
      sp.pp = (int)rawpp.size();
      make_prim_pairs(c, a, b, rawpp);
      sp.npp = (int)rawpp.size() - sp.pp;
      sp.Q = 0.0;
      sp.diag = (a == b);
      sp.cls = pair_class(c->l[a], c->l[b]);
      ids[sp.cls].push_back((int)raw.size());
      raw.push_back(sp);
    }
  c->n_pairs_all = (long long)raw.size();
  // 2. Schwarz bounds on the device
  DevBuf<ShellPair> d_raw;
  DevBuf<PrimPair> d_rawpp;
  DevBuf<unsigned long long> d_q;
  DevBuf<int> d_ids;
  JQC_CUDA_CHECK(d_raw.upload(raw, s));
  JQC_CUDA_CHECK(d_rawpp.upload(rawpp, s));
  JQC_CUDA_CHECK(d_q.reserve(raw.size()));
  JQC_CUDA_CHECK(cudaMemsetAsync(d_q.ptr, 0, raw.size() * sizeof(unsigned long long), s));
  std::vector<int> all_ids;
  int id_off[kNumPairClasses];
  for (int pc = 0; pc < kNumPairClasses; ++pc) {
    id_off[pc] = (int)all_ids.size();
    all_ids.insert(all_ids.end(), ids[pc].begin(), ids[pc].end());
  }
  JQC_CUDA_CHECK(d_ids.upload(all_ids, s));
  for (int pc = 0; pc < kNumPairClasses; ++pc) {
    SchwarzParams p;
    p.pair_ids = d_ids.ptr + id_off[pc];
    p.n_pairs = (int)ids[pc].size();
    p.pairs = d_raw.ptr;
    p.pp = d_rawpp.ptr;
    p.centres = c->d_centres.ptr;
    p.boys = c->boys64;
    p.boys_al = c->boysA64;
    p.qmax = d_q.ptr;
    JQC_CUDA_CHECK(launch_schwarz(pc, p, s));
  }
  std::vector<unsigned long long> qbits(raw.size());
  JQC_CUDA_CHECK(cudaMemcpyAsync(qbits.data(), d_q.ptr, qbits.size() * sizeof(unsigned long long),
                                 cudaMemcpyDeviceToHost, s));
  JQC_CUDA_CHECK(cudaStreamSynchronize(s));
  std::vector<double> qmax(c->n_mol, 0.0);  // largest Q of each molecule
  c->Qmat.assign((size_t)c->n_shell * c->n_shell, 0.0);
  for (size_t k = 0; k < raw.size(); ++k) {
    double v;
    std::memcpy(&v, &qbits[k], sizeof(double));
    raw[k].Q = std::sqrt(std::max(v, 0.0));
    double& qm = qmax[c->shell_mol[raw[k].a]];
    qm = std::max(qm, raw[k].Q);
    c->Qmat[(size_t)raw[k].a * c->n_shell + raw[k].b] = raw[k].Q;
    c->Qmat[(size_t)raw[k].b * c->n_shell + raw[k].a] = raw[k].Q;
  }
  // 3. drop pairs that cannot pass with any pair of their molecule, sort by
  // (class, primitive pairs, molecule) then Q descending
  std::vector<int> keep;
  for (size_t k = 0; k < raw.size(); ++k)
    if (raw[k].Q * qmax[c->shell_mol[raw[k].a]] >= schwarz_tau && raw[k].Q > 0.0) keep.push_back((int)k);
  auto key = [&](int k) {
    const ShellPair& p = raw[k];
    return std::make_tuple(p.cls, p.npp, c->shell_mol[p.a]);
  };
  std::stable_sort(keep.begin(), keep.end(), [&](int x, int y) {
    auto kx = key(x), ky = key(y);
    if (kx != ky) return kx < ky;
    return raw[x].Q > raw[y].Q;
  });
  c->pairs.clear();
  c->blocks.clear();
  std::vector<PrimPair> pp;
  std::vector<PrimPairF> ppf;
  for (size_t r = 0; r < keep.size(); ++r) {
    ShellPair sp = raw[keep[r]];
    const int src = sp.pp;
    sp.pp = (int)pp.size();
    for (int k = 0; k < sp.npp; ++k) {
      const PrimPair& q = rawpp[src + k];
      pp.push_back(q);
      ppf.push_back(PrimPairF{float(q.p), float(q.h), float(q.Px), float(q.Py), float(q.Pz), float(q.K),
                              float(q.alpha), float(q.beta)});
    }
    auto kk = key(keep[r]);
    if (c->blocks.empty() || std::get<0>(kk) != c->blocks.back().pc || std::get<1>(kk) != c->blocks.back().ka ||
        std::get<2>(kk) != c->blocks.back().mol) {
      c->blocks.push_back(Block{std::get<0>(kk), std::get<1>(kk), 1, (int)c->pairs.size(), 0, std::get<2>(kk)});
    }
    c->blocks.back().count++;
    c->pairs.push_back(sp);
  }
  JQC_CUDA_CHECK(c->d_pairs.upload(c->pairs, s));
  JQC_CUDA_CHECK(c->d_pp.upload(pp, s));
  JQC_CUDA_CHECK(c->d_ppf.upload(ppf, s));
  JQC_CUDA_CHECK(cudaStreamSynchronize(s));
  c->tau = schwarz_tau;
  c->pairs_ready = true;
  drop_jk_tasks(c);
  c->full_tasks.valid = false;
  c->grad_tasks.valid = false;
  return JQC_OK;
}

int jqc_stats(jqc_ctx* c, int precision_mode, double mixed_tau, long long* out) {
  JQC_REQUIRE(c && out, JQC_ERR_INVALID, "jqc_stats: null argument");
  JQC_REQUIRE(c->pairs_ready, JQC_ERR_NOT_READY, "jqc_stats: call jqc_pairs_build first");
  JQC_REQUIRE(precision_mode >= 0 && precision_mode <= 2, JQC_ERR_INVALID, "jqc_stats: bad precision_mode");
  int rc = select_device(c);
  if (rc) return rc;
  rc = ensure_jk_tasks(c, precision_mode, mixed_tau, 0);
  if (rc) return rc;
  JQC_CUDA_CHECK(cudaStreamSynchronize(0));
  out[0] = c->n_pairs_all;
  out[1] = (long long)c->pairs.size();
  out[2] = c->jk_cur->n_quartets[0];
  out[3] = c->jk_cur->n_quartets[1];
  out[4] = c->jk_cur->n_prim_quartets;
  out[5] = c->n_bf;
  int launches = 2;  // J and K symmetrization
  for (int prec = 0; prec < 2; ++prec)
    for (int qc = 0; qc < kNumQuartetClasses; ++qc) launches += c->jk_cur->cnt[prec][qc] > 0;
  out[6] = (long long)c->jk_cur->h.size();
  out[7] = launches;
  return JQC_OK;
}

int jqc_class_stats(jqc_ctx* c, int precision_mode, double mixed_tau, long long* out) {
  JQC_REQUIRE(c && out, JQC_ERR_INVALID, "jqc_class_stats: null argument");
  JQC_REQUIRE(c->pairs_ready, JQC_ERR_NOT_READY, "jqc_class_stats: call jqc_pairs_build first");
  JQC_REQUIRE(precision_mode >= 0 && precision_mode <= 2, JQC_ERR_INVALID, "jqc_class_stats: bad precision_mode");
  int rc = select_device(c);
  if (rc) return rc;
  rc = ensure_jk_tasks(c, precision_mode, mixed_tau, 0);
  if (rc) return rc;
  for (int prec = 0; prec < 2; ++prec)
    for (int qc = 0; qc < kNumQuartetClasses; ++qc) {
      const int k = (prec * kNumQuartetClasses + qc) * 3;
      out[k] = c->jk_cur->class_quartets[prec][qc];
      out[k + 1] = c->jk_cur->class_prims[prec][qc];
      out[k + 2] = c->jk_cur->cnt[prec][qc];
    }
  return JQC_OK;
}

int jqc_fp_peak(int fp32, int blocks, int iters, double* tflops, void* stream) {
  JQC_REQUIRE(tflops != nullptr && blocks > 0 && iters > 0, JQC_ERR_INVALID, "jqc_fp_peak: bad argument");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  void* sink = nullptr;
  JQC_CUDA_CHECK(cudaMalloc(&sink, (size_t)blocks * 8));
  float ms = 0.f;
  cudaError_t e = fma_peak(fp32 != 0, blocks, iters, sink, s, &ms);
  cudaFree(sink);
  JQC_CUDA_CHECK(e);
  const double flops = 2.0 * 8 * 16 * (double)iters * 256.0 * blocks;
  *tflops = flops / (ms * 1e-3) / 1e12;
  return JQC_OK;
}

int jqc_schwarz(jqc_ctx* c, double* Q, void* stream) {
  JQC_REQUIRE(c && Q, JQC_ERR_INVALID, "jqc_schwarz: null argument");
  JQC_REQUIRE(c->pairs_ready, JQC_ERR_NOT_READY, "jqc_schwarz: call jqc_pairs_build first");
  int rc = select_device(c);
  if (rc) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  JQC_CUDA_CHECK(cudaMemcpyAsync(Q, c->Qmat.data(), c->Qmat.size() * sizeof(double), cudaMemcpyHostToDevice, s));
  JQC_CUDA_CHECK(cudaStreamSynchronize(s));
  return JQC_OK;
}

int jqc_boys(const double* T, long long n, int mmax, void* out, int fp32, void* stream) {
  JQC_REQUIRE(n >= 0, JQC_ERR_INVALID, "jqc_boys: n must be >= 0");
  JQC_REQUIRE(mmax >= 0 && mmax <= kBoysMaxM, JQC_ERR_INVALID, "jqc_boys: mmax must be in [0, 16]");
  if (n == 0) return JQC_OK;
  JQC_REQUIRE(T && out, JQC_ERR_INVALID, "jqc_boys: null pointer");
  int dev = 0;
  JQC_CUDA_CHECK(cudaGetDevice(&dev));
  BoysTables bt;
  int rc = boys_tables_all(dev, &bt);
  if (rc) return rc;
  JQC_CUDA_CHECK(launch_boys(T, n, mmax, out, fp32 != 0, fp32 ? (const void*)bt.a32 : (const void*)bt.a64,
                             static_cast<cudaStream_t>(stream)));
  return JQC_OK;
}

int jqc_eri_prim_quartets(int la, int lb, int lc, int ld, long long n, const double* exps, const double* centres,
                          double* out, void* stream) {
  JQC_REQUIRE(n >= 0, JQC_ERR_INVALID, "jqc_eri_prim_quartets: n must be >= 0");
  JQC_REQUIRE(la >= 0 && lb >= 0 && lc >= 0 && ld >= 0, JQC_ERR_INVALID, "jqc_eri_prim_quartets: negative l");
  JQC_REQUIRE(la <= kMaxL && lb <= kMaxL && lc <= kMaxL && ld <= kMaxL, JQC_ERR_UNSUPPORTED,
              "jqc_eri_prim_quartets: l > 2 is not supported");
  JQC_REQUIRE(la >= lb && lc >= ld && pair_class(la, lb) >= pair_class(lc, ld), JQC_ERR_UNSUPPORTED,
              "jqc_eri_prim_quartets: class must satisfy la>=lb, lc>=ld, (la,lb)>=(lc,ld)");
  if (n == 0) return JQC_OK;
  JQC_REQUIRE(exps && centres && out, JQC_ERR_INVALID, "jqc_eri_prim_quartets: null pointer");
  int dev = 0;
  JQC_CUDA_CHECK(cudaGetDevice(&dev));
  BoysTables bt;
  int rc = boys_tables_all(dev, &bt);
  if (rc) return rc;
  PrimQuartetParams p{n, exps, centres, bt.t64, bt.a64, out};
  JQC_CUDA_CHECK(launch_prim_quartets(la, lb, lc, ld, p, static_cast<cudaStream_t>(stream)));
  return JQC_OK;
}

int jqc_eri_tensor(jqc_ctx* c, double* out, long long max_bytes, void* stream) {
  JQC_REQUIRE(c && out, JQC_ERR_INVALID, "jqc_eri_tensor: null argument");
  JQC_REQUIRE(c->pairs_ready, JQC_ERR_NOT_READY, "jqc_eri_tensor: call jqc_pairs_build first");
  const double bytes = std::pow((double)c->n_bf, 4) * 8.0;
  JQC_REQUIRE(bytes <= (double)max_bytes, JQC_ERR_TOO_LARGE,
              "jqc_eri_tensor: n^4 tensor exceeds max_bytes; use jqc_jk (direct J/K) instead");
  int rc = select_device(c);
  if (rc) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  JQC_REQUIRE(!stream_capturing(s), JQC_ERR_INVALID, "jqc_eri_tensor: cannot run inside a graph capture");
  rc = ensure_tasks(c, c->full_tasks, JQC_PREC_FP64, 0.0, true, s);
  if (rc) return rc;
  JQC_CUDA_CHECK(cudaMemsetAsync(out, 0, (size_t)bytes, s));
  for (int qc = 0; qc < kNumQuartetClasses; ++qc) {
    TensorParams p;
    p.tasks = c->full_tasks.d.ptr + c->full_tasks.off[0][qc];
    p.n_tasks = c->full_tasks.cnt[0][qc];
    p.pairs = c->d_pairs.ptr;
    p.pp = c->d_pp.ptr;
    p.centres = c->d_centres.ptr;
    p.ao = c->d_ao.ptr;
    p.boys = c->boys64;
    p.boys_al = c->boysA64;
    p.eri = out;
    p.n = c->n_bf;
    JQC_CUDA_CHECK(launch_eri_tensor(qc, p, s));
  }
  return JQC_OK;
}

int jqc_grad2e_ex(jqc_ctx* c, int n_dens, const double* D, double j_scale, double k_scale, double dens_tau,
                  double* grad, void* stream, double* class_ms) {
  JQC_REQUIRE(c && D && grad, JQC_ERR_INVALID, "jqc_grad2e: null argument");
  JQC_REQUIRE(n_dens >= 1 && n_dens <= 4, JQC_ERR_INVALID, "jqc_grad2e: n_dens must be 1..4");
  JQC_REQUIRE(c->pairs_ready, JQC_ERR_NOT_READY, "jqc_grad2e: call jqc_pairs_build first");
  JQC_REQUIRE(c->n_atom > 0, JQC_ERR_NOT_READY, "jqc_grad2e: the basis was uploaded without atoms");
  JQC_REQUIRE(dens_tau >= 0.0 && std::isfinite(dens_tau), JQC_ERR_INVALID, "jqc_grad2e: dens_tau must be >= 0");
  int rc = select_device(c);
  if (rc) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const bool capturing = stream_capturing(s);
  JQC_REQUIRE(!(capturing && class_ms), JQC_ERR_INVALID, "jqc_grad2e_ex: timing cannot run inside a graph capture");
  JQC_REQUIRE(c->grad_tasks.valid || !capturing, JQC_ERR_NOT_READY,
              "jqc_grad2e: no gradient work list; call jqc_grad2e once before the capture");
  JQC_REQUIRE(dens_tau <= 0.0 || !capturing || c->d_dmax.n >= (size_t)c->n_shell * c->n_shell + 1, JQC_ERR_NOT_READY,
              "jqc_grad2e: density screening scratch not allocated; call once before the capture");
  if (!c->grad_tasks.valid) {
    rc = build_tasks(c, c->grad_tasks, JQC_PREC_FP64, 0.0, false, s, true);
    if (rc) return rc;
  }
  const float* dmax = nullptr;
  float* dmax_top = nullptr;
  if (dens_tau > 0.0) {
    JQC_CUDA_CHECK(c->d_dmax.reserve((size_t)c->n_shell * c->n_shell + 1));
    dmax_top = c->d_dmax.ptr + (size_t)c->n_shell * c->n_shell;
    JQC_CUDA_CHECK(
        launch_dmax(D, n_dens, c->n_bf, c->n_shell, c->d_ao.ptr, c->d_l.ptr, c->d_dmax.ptr, dmax_top, s));
    dmax = c->d_dmax.ptr;
  }
  const int n_pairs = (int)c->pairs.size();
  JQC_REQUIRE(!capturing || c->d_pair_force.n >= (size_t)6 * n_pairs, JQC_ERR_NOT_READY,
              "jqc_grad2e: force scratch not allocated; call jqc_grad2e once before the capture");
  JQC_CUDA_CHECK(c->d_pair_force.reserve((size_t)6 * std::max(1, n_pairs)));
  JQC_CUDA_CHECK(cudaMemsetAsync(c->d_pair_force.ptr, 0, (size_t)6 * n_pairs * sizeof(double), s));
  if (class_ms)
    for (int k = 0; k < kNumQuartetClasses; ++k) class_ms[k] = 0.0;
  for (int qc = 0; qc < kNumQuartetClasses; ++qc) {
    GradParams p;
    p.tasks = c->grad_tasks.d.ptr + c->grad_tasks.off[0][qc];
    p.n_tasks = c->grad_tasks.cnt[0][qc];
    if (p.n_tasks == 0) continue;
    p.pairs = c->d_pairs.ptr;
    p.pp = c->d_pp.ptr;
    p.centres = c->d_centres.ptr;
    p.ao = c->d_ao.ptr;
    p.atom = c->d_atom.ptr;
    p.boys = c->boys64;
    p.boys_al = c->boysA64;
    p.D = D;
    p.n_dens = n_dens;
    p.n = c->n_bf;
    p.jscale = j_scale;
    p.kscale = k_scale;
    p.grad = grad;
    p.pair_force = c->d_pair_force.ptr;
    p.dmax = dmax;
    p.dmax_top = dmax_top;
    p.n_shell = c->n_shell;
    p.dens_tau = (float)dens_tau;
    const int pb = qc_bra(qc), pk = qc_ket(qc);
    if (class_ms) JQC_CUDA_CHECK(cudaEventRecord(c->ev_t0, s));
    const int ge = c->grad_engine[qc];
    p.sides = ge == kGradEngineRegSplit ? 2 : 1;
    if (grad_reg_engine(ge))
      JQC_CUDA_CHECK(launch_grad_reg(qc, p, s));
    else if (ge == kEngineCol)
      JQC_CUDA_CHECK(launch_grad_row(qc, p, s));
    else
      JQC_CUDA_CHECK(launch_warp_grad(pc_la(pb), pc_lb(pb), pc_la(pk), pc_lb(pk), p, s));
    if (class_ms) {
      JQC_CUDA_CHECK(cudaEventRecord(c->ev_t1, s));
      JQC_CUDA_CHECK(cudaEventSynchronize(c->ev_t1));
      float ms = 0.f;
      JQC_CUDA_CHECK(cudaEventElapsedTime(&ms, c->ev_t0, c->ev_t1));
      class_ms[qc] = ms;
    }
  }
  JQC_CUDA_CHECK(launch_pair_force_reduce(c->d_pairs.ptr, n_pairs, c->d_atom.ptr, c->d_pair_force.ptr, grad, s));
  return JQC_OK;
}

int jqc_grad2e(jqc_ctx* c, int n_dens, const double* D, double j_scale, double k_scale, double* grad,
               void* stream) {
  return jqc_grad2e_ex(c, n_dens, D, j_scale, k_scale, 0.0, grad, stream, nullptr);
}

int jqc_grad1e(jqc_ctx* c, const double* D, const double* W, double* grad, void* stream) {
  JQC_REQUIRE(c && D && W && grad, JQC_ERR_INVALID, "jqc_grad1e: null argument");
  JQC_REQUIRE(c->basis_ready, JQC_ERR_NOT_READY, "jqc_grad1e: call jqc_basis_upload first");
  JQC_REQUIRE(c->n_atom > 0, JQC_ERR_NOT_READY, "jqc_grad1e: the basis was uploaded without atoms");
  int rc = select_device(c);
  if (rc) return rc;
  Grad1Params p;
  p.n_shell = c->n_shell;
  p.n = c->n_bf;
  p.n_atom = c->n_atom;
  p.l = c->d_l.ptr;
  p.nprim = c->d_nprim.ptr;
  p.prim_off = c->d_prim_off.ptr;
  p.exps = c->d_exps.ptr;
  p.coefs = c->d_coefs.ptr;
  p.centres = c->d_centres.ptr;
  p.ao = c->d_ao.ptr;
  p.atom = c->d_atom.ptr;
  p.atom_xyz = c->d_atom_xyz.ptr;
  p.atom_Z = c->d_atom_Z.ptr;
  p.shell_mol = c->n_mol > 1 ? c->d_shell_mol.ptr : nullptr;
  p.atom_mol = c->n_mol > 1 ? c->d_atom_mol.ptr : nullptr;
  p.boys = c->boys64;
  p.boys_al = c->boysA64;
  p.D = D;
  p.W = W;
  p.grad = grad;
  JQC_CUDA_CHECK(launch_grad1e(p, static_cast<cudaStream_t>(stream)));
  return JQC_OK;
}

int jqc_one_electron(jqc_ctx* c, double* S, double* T, double* V, void* stream) {
  JQC_REQUIRE(c && S && T && V, JQC_ERR_INVALID, "jqc_one_electron: null argument");
  JQC_REQUIRE(c->basis_ready, JQC_ERR_NOT_READY, "jqc_one_electron: call jqc_basis_upload first");
  int rc = select_device(c);
  if (rc) return rc;
  OneEParams p;
  p.n_shell = c->n_shell;
  p.n = c->n_bf;
  p.n_atom = c->n_atom;
  p.l = c->d_l.ptr;
  p.nprim = c->d_nprim.ptr;
  p.prim_off = c->d_prim_off.ptr;
  p.exps = c->d_exps.ptr;
  p.coefs = c->d_coefs.ptr;
  p.centres = c->d_centres.ptr;
  p.ao = c->d_ao.ptr;
  p.atom_xyz = c->d_atom_xyz.ptr;
  p.atom_Z = c->d_atom_Z.ptr;
  p.shell_mol = c->n_mol > 1 ? c->d_shell_mol.ptr : nullptr;
  p.atom_mol = c->n_mol > 1 ? c->d_atom_mol.ptr : nullptr;
  p.boys = c->boys64;
  p.S = S;
  p.T = T;
  p.V = V;
  JQC_CUDA_CHECK(launch_one_e(p, static_cast<cudaStream_t>(stream)));
  return JQC_OK;
}

static int jk_impl(jqc_ctx* c, int n_dens, const double* D, double* J, double* K, int precision_mode,
                   double mixed_tau, double dens_tau, cudaStream_t s, double* class_ms);

int jqc_jk_timed(jqc_ctx* c, int n_dens, const double* D, double* J, double* K, int precision_mode, double mixed_tau,
                 double dens_tau, void* stream, double* class_ms) {
  JQC_REQUIRE(class_ms != nullptr, JQC_ERR_INVALID, "jqc_jk_timed: class_ms is null");
  return jk_impl(c, n_dens, D, J, K, precision_mode, mixed_tau, dens_tau, static_cast<cudaStream_t>(stream),
                 class_ms);
}

int jqc_jk(jqc_ctx* c, int n_dens, const double* D, double* J, double* K, int precision_mode, double mixed_tau,
           double dens_tau, void* stream) {
  return jk_impl(c, n_dens, D, J, K, precision_mode, mixed_tau, dens_tau, static_cast<cudaStream_t>(stream),
                 nullptr);
}

static int jk_impl(jqc_ctx* c, int n_dens, const double* D, double* J, double* K, int precision_mode,
                   double mixed_tau, double dens_tau, cudaStream_t s, double* class_ms) {
  JQC_REQUIRE(c && D && J && K, JQC_ERR_INVALID, "jqc_jk: null argument");
  JQC_REQUIRE(n_dens >= 1 && n_dens <= 4, JQC_ERR_INVALID, "jqc_jk: n_dens must be 1..4");
  JQC_REQUIRE(c->pairs_ready, JQC_ERR_NOT_READY, "jqc_jk: call jqc_pairs_build first");
  JQC_REQUIRE(precision_mode >= 0 && precision_mode <= 2, JQC_ERR_INVALID, "jqc_jk: bad precision_mode");
  JQC_REQUIRE(mixed_tau >= 0.0 && dens_tau >= 0.0, JQC_ERR_INVALID, "jqc_jk: thresholds must be >= 0");
  int rc = select_device(c);
  if (rc) return rc;
  const bool capturing = stream_capturing(s);
  JQC_REQUIRE(!(capturing && class_ms), JQC_ERR_INVALID, "jqc_jk_timed: cannot run inside a graph capture");
  if (capturing) {
    // inside a capture nothing may be allocated or uploaded
    JQC_REQUIRE(find_jk_tasks(c, precision_mode, mixed_tau) != nullptr, JQC_ERR_NOT_READY,
                "jqc_jk: no work list for this precision_mode/mixed_tau; call jqc_jk once before the capture");
    JQC_REQUIRE(dens_tau <= 0.0 || c->d_dmax.n >= (size_t)c->n_shell * c->n_shell + 1, JQC_ERR_NOT_READY,
                "jqc_jk: density screening scratch not allocated; call jqc_jk once before the capture");
  }
  rc = ensure_jk_tasks(c, precision_mode, mixed_tau, s);
  if (rc) return rc;
  float* dmax = nullptr;
  float* dmax_top = nullptr;
  if (dens_tau > 0.0) {
    JQC_CUDA_CHECK(c->d_dmax.reserve((size_t)c->n_shell * c->n_shell + 1));
    dmax = c->d_dmax.ptr;
    dmax_top = dmax + (size_t)c->n_shell * c->n_shell;
  }
  return run_jk_set(c, c->jk_cur, n_dens, D, J, K, dmax, dmax_top, dens_tau, s, class_ms);
}

// ----------------------------------------------------------- CUDA graphs
int jqc_graph_begin(jqc_ctx* c, void* stream) {
  JQC_REQUIRE(c != nullptr, JQC_ERR_INVALID, "jqc_graph_begin: null context");
  JQC_REQUIRE(stream != nullptr, JQC_ERR_INVALID,
              "jqc_graph_begin: the legacy default stream cannot be captured; pass a created stream");
  int rc = select_device(c);
  if (rc) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  JQC_REQUIRE(!stream_capturing(s), JQC_ERR_INVALID, "jqc_graph_begin: the stream is already capturing");
  JQC_CUDA_CHECK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  return JQC_OK;
}

int jqc_graph_end(jqc_ctx* c, void* stream, int* graph_id) {
  JQC_REQUIRE(c && graph_id, JQC_ERR_INVALID, "jqc_graph_end: null argument");
  int rc = select_device(c);
  if (rc) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaGraph_t g = nullptr;
  JQC_CUDA_CHECK(cudaStreamEndCapture(s, &g));
  JQC_REQUIRE(g != nullptr, JQC_ERR_CUDA, "jqc_graph_end: the capture produced no graph");
  cudaGraphExec_t ex = nullptr;
  cudaError_t e = cudaGraphInstantiate(&ex, g, 0);
  cudaGraphDestroy(g);
  JQC_CUDA_CHECK(e);
  c->graphs.push_back(ex);
  *graph_id = (int)c->graphs.size() - 1;
  return JQC_OK;
}

int jqc_graph_launch(jqc_ctx* c, int graph_id, void* stream) {
  JQC_REQUIRE(c != nullptr, JQC_ERR_INVALID, "jqc_graph_launch: null context");
  JQC_REQUIRE(graph_id >= 0 && graph_id < (int)c->graphs.size() && c->graphs[graph_id], JQC_ERR_INVALID,
              "jqc_graph_launch: unknown graph id, or the graph was invalidated by a new basis, pair list, "
              "work list or tuning");
  int rc = select_device(c);
  if (rc) return rc;
  JQC_CUDA_CHECK(cudaGraphLaunch(c->graphs[graph_id], static_cast<cudaStream_t>(stream)));
  return JQC_OK;
}

int jqc_graph_destroy(jqc_ctx* c, int graph_id) {
  JQC_REQUIRE(c != nullptr, JQC_ERR_INVALID, "jqc_graph_destroy: null context");
  JQC_REQUIRE(graph_id >= 0 && graph_id < (int)c->graphs.size(), JQC_ERR_INVALID,
              "jqc_graph_destroy: unknown graph id");
  int rc = select_device(c);
  if (rc) return rc;
  if (c->graphs[graph_id]) JQC_CUDA_CHECK(cudaGraphExecDestroy(c->graphs[graph_id]));
  c->graphs[graph_id] = nullptr;
  return JQC_OK;
}

// ------------------------------------------------------------ autotuning
int jqc_get_tuning(jqc_ctx* c, int* out) {
  JQC_REQUIRE(c && out, JQC_ERR_INVALID, "jqc_get_tuning: null argument");
  for (int qc = 0; qc < kNumQuartetClasses; ++qc) {
    out[kTuneInts * qc] = c->tune[qc].threads;
    out[kTuneInts * qc + 1] = c->tune[qc].lane_prims;
    out[kTuneInts * qc + 2] = c->tune[qc].persistent;
    out[kTuneInts * qc + 3] = class_engine(c->tune[qc], qc);
  }
  return JQC_OK;
}

int jqc_set_tuning(jqc_ctx* c, const int* cfg) {
  JQC_REQUIRE(c && cfg, JQC_ERR_INVALID, "jqc_set_tuning: null argument");
  for (int qc = 0; qc < kNumQuartetClasses; ++qc) {
    const int* q = cfg + kTuneInts * qc;
    JQC_REQUIRE(q[0] == 64 || q[0] == 128 || q[0] == 256, JQC_ERR_INVALID,
                "jqc_set_tuning: threads must be 64, 128 or 256");
    JQC_REQUIRE(q[1] >= 1 && q[1] <= (1 << 20), JQC_ERR_INVALID, "jqc_set_tuning: lane_prims out of range");
    JQC_REQUIRE(q[2] == 0 || q[2] == 1, JQC_ERR_INVALID, "jqc_set_tuning: persistent must be 0 or 1");
    JQC_REQUIRE(engine_valid(q[3], qc), JQC_ERR_INVALID,
                "jqc_set_tuning: engine must be 0 (register, L <= 6), 1 (column, L >= 5) or 2 (warp)");
  }
  bool lists_changed = false;
  for (int qc = 0; qc < kNumQuartetClasses; ++qc) {
    const int* q = cfg + kTuneInts * qc;
    const bool per_task_changed = (class_engine(c->tune[qc], qc) == kEngineReg) != (q[3] == kEngineReg);
    if (c->tune[qc].lane_prims != q[1] || per_task_changed) lists_changed = true;
    c->tune[qc] = ClassTune{q[0], q[1], q[2], q[3]};
  }
  if (lists_changed) drop_jk_tasks(c);  // the work lists depend on lane_prims and the engine
  return JQC_OK;
}

int jqc_set_grad_engine(jqc_ctx* c, int quartet_class, int engine) {
  JQC_REQUIRE(c != nullptr, JQC_ERR_INVALID, "jqc_set_grad_engine: null context");
  JQC_REQUIRE(quartet_class >= 0 && quartet_class < kNumQuartetClasses, JQC_ERR_INVALID,
              "jqc_set_grad_engine: quartet class out of range");
  JQC_REQUIRE(grad_engine_valid(engine, quartet_class), JQC_ERR_INVALID,
              "jqc_set_grad_engine: engine must be 0 (register, L <= 4), 1 (row, dp/dd bra), 2 (warp) or "
              "3 (register, bra and ket forces in separate parts, L <= 4)");
  const bool per_task_changed = grad_reg_engine(c->grad_engine[quartet_class]) != grad_reg_engine(engine);
  c->grad_engine[quartet_class] = engine;
  if (per_task_changed && c->grad_tasks.valid) {
    drop_graphs(c);
    c->grad_tasks.valid = false;
  }
  return JQC_OK;
}

int jqc_get_grad_engine(jqc_ctx* c, int* engines21) {
  JQC_REQUIRE(c && engines21, JQC_ERR_INVALID, "jqc_get_grad_engine: null argument");
  for (int qc = 0; qc < kNumQuartetClasses; ++qc) engines21[qc] = c->grad_engine[qc];
  return JQC_OK;
}

// Workload signature for the tuning cache: device, precision settings and
// the order of magnitude of the screened quartets of every class.
static std::string tune_signature(jqc_ctx* c, const TaskSet* ts, int n_dens, int precision_mode, double dens_tau) {
  cudaDeviceProp prop;
  std::string sig = "jqc-tune1";
  if (cudaGetDeviceProperties(&prop, c->device) == cudaSuccess) {
    std::string name = prop.name;
    for (char& ch : name)
      if (ch == ' ' || ch == '\t') ch = '_';
    sig += " dev=" + name + "/" + std::to_string(prop.multiProcessorCount);
  }
  sig += " mode=" + std::to_string(precision_mode) + " ndens=" + std::to_string(n_dens) +
         " dscreen=" + std::to_string(dens_tau > 0.0 ? 1 : 0) + " q=";
  for (int prec = 0; prec < 2; ++prec)
    for (int qc = 0; qc < kNumQuartetClasses; ++qc) {
      const long long q = ts->class_quartets[prec][qc];
      sig += std::to_string(q > 0 ? std::ilogb((double)q) + 1 : 0);
      sig += (prec == 1 && qc == kNumQuartetClasses - 1) ? "" : ",";
    }
  return sig;
}

int jqc_autotune(jqc_ctx* c, int n_dens, const double* D, double* J, double* K, int precision_mode, double mixed_tau,
                 double dens_tau, const char* cache_path, int* from_cache, void* stream) {
  JQC_REQUIRE(c && D && J && K, JQC_ERR_INVALID, "jqc_autotune: null argument");
  JQC_REQUIRE(n_dens >= 1 && n_dens <= 4, JQC_ERR_INVALID, "jqc_autotune: n_dens must be 1..4");
  JQC_REQUIRE(c->pairs_ready, JQC_ERR_NOT_READY, "jqc_autotune: call jqc_pairs_build first");
  JQC_REQUIRE(precision_mode >= 0 && precision_mode <= 2, JQC_ERR_INVALID, "jqc_autotune: bad precision_mode");
  JQC_REQUIRE(mixed_tau >= 0.0 && dens_tau >= 0.0, JQC_ERR_INVALID, "jqc_autotune: thresholds must be >= 0");
  int rc = select_device(c);
  if (rc) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  JQC_REQUIRE(!stream_capturing(s), JQC_ERR_INVALID, "jqc_autotune: cannot run inside a graph capture");
  if (from_cache) *from_cache = 0;
  rc = ensure_jk_tasks(c, precision_mode, mixed_tau, s);
  if (rc) return rc;
  const std::string sig = tune_signature(c, c->jk_cur, n_dens, precision_mode, dens_tau);
  int cfg[kTuneInts * kNumQuartetClasses];
  // 1. cache hit: "signature<TAB>84 integers" per line
  if (cache_path && cache_path[0]) {
    std::FILE* f = std::fopen(cache_path, "r");
    if (f) {
      std::string line;
      bool hit = false;
      int ch;
      while (!hit) {
        line.clear();
        while ((ch = std::fgetc(f)) != EOF && ch != '\n') line.push_back((char)ch);
        const size_t tab = line.find('\t');
        if (tab != std::string::npos && line.compare(0, tab, sig) == 0 && tab == sig.size()) {
          const char* q = line.c_str() + tab + 1;
          int k = 0;
          char* end = nullptr;
          for (; k < kTuneInts * kNumQuartetClasses; ++k) {
            const long v = std::strtol(q, &end, 10);
            if (end == q) break;
            cfg[k] = (int)v;
            q = end;
          }
          hit = (k == kTuneInts * kNumQuartetClasses);
        }
        if (ch == EOF) break;
      }
      std::fclose(f);
      if (hit) {
        rc = jqc_set_tuning(c, cfg);
        if (rc) return rc;
        rc = ensure_jk_tasks(c, precision_mode, mixed_tau, s);
        if (rc) return rc;
        if (from_cache) *from_cache = 1;
        return JQC_OK;
      }
    }
  }
  float* dmax = nullptr;
  float* dmax_top = nullptr;
  if (dens_tau > 0.0) {
    JQC_CUDA_CHECK(c->d_dmax.reserve((size_t)c->n_shell * c->n_shell + 1));
    dmax = c->d_dmax.ptr;
    dmax_top = dmax + (size_t)c->n_shell * c->n_shell;
  }
  // per-class time of the current settings: min over two timed builds, or
  // one when a build takes long enough (> 30 ms) for one to be steady
  double ms[2 * kNumQuartetClasses], best_ms[kNumQuartetClasses];
  auto time_classes = [&](double* per_class) -> int {
    for (int qc = 0; qc < kNumQuartetClasses; ++qc) per_class[qc] = 1e300;
    for (int rep = 0; rep < 2; ++rep) {
      int r = run_jk_set(c, c->jk_cur, n_dens, D, J, K, dmax, dmax_top, dens_tau, s, ms);
      if (r) return r;
      double total = 0.0;
      for (int qc = 0; qc < kNumQuartetClasses; ++qc) {
        per_class[qc] = std::min(per_class[qc], ms[qc] + ms[kNumQuartetClasses + qc]);
        total += ms[qc] + ms[kNumQuartetClasses + qc];
      }
      if (total > 30.0) break;
    }
    return JQC_OK;
  };
  ClassTune best[kNumQuartetClasses];
  for (int qc = 0; qc < kNumQuartetClasses; ++qc) {
    best[qc] = ClassTune{};
    best[qc].engine = default_engine(qc);
    best_ms[qc] = 1e300;
  }
  double cur[kNumQuartetClasses];
  auto rebuild = [&]() -> int {
    drop_jk_tasks(c);
    return ensure_jk_tasks(c, precision_mode, mixed_tau, s);
  };
  // 2. engine of every class, register or column kernels where a class has
  // both (the runtime-class warp engine is never the faster one; it stays
  // the fallback of classes without either)
  for (int e = kEngineReg; e <= kEngineCol; ++e) {
    for (int qc = 0; qc < kNumQuartetClasses; ++qc)
      c->tune[qc] = ClassTune{128, kMaxLanePrims, 0, engine_valid(e, qc) ? e : default_engine(qc)};
    rc = rebuild();
    if (rc) return rc;
    rc = time_classes(cur);
    if (rc) return rc;
    for (int qc = 0; qc < kNumQuartetClasses; ++qc)
      if (engine_valid(e, qc) && cur[qc] < best_ms[qc]) {
        best_ms[qc] = cur[qc];
        best[qc].engine = e;
      }
  }
  for (int qc = 0; qc < kNumQuartetClasses; ++qc) c->tune[qc] = ClassTune{128, kMaxLanePrims, 0, best[qc].engine};
  rc = rebuild();
  if (rc) return rc;
  // 3. block size and grid form of the register kernels (no rebuild needed)
  const int th_opts[2] = {128, 256};
  for (int ti = 0; ti < 2; ++ti)
    for (int pe = 0; pe < 2; ++pe) {
      for (int qc = 0; qc < kNumQuartetClasses; ++qc) {
        c->tune[qc].threads = th_opts[ti];
        c->tune[qc].persistent = pe;
      }
      rc = time_classes(cur);
      if (rc) return rc;
      for (int qc = 0; qc < kNumQuartetClasses; ++qc)
        if (best[qc].engine == kEngineReg && cur[qc] < best_ms[qc]) {
          best_ms[qc] = cur[qc];
          best[qc].threads = th_opts[ti];
          best[qc].persistent = pe;
        }
    }
  // 4. bra primitive chunk (work list rebuilt per value)
  const int lp_opts[3] = {64, 128, 512};
  for (int qc = 0; qc < kNumQuartetClasses; ++qc) {
    c->tune[qc].threads = best[qc].threads;
    c->tune[qc].persistent = best[qc].persistent;
  }
  for (int li = 0; li < 3; ++li) {
    for (int qc = 0; qc < kNumQuartetClasses; ++qc) c->tune[qc].lane_prims = lp_opts[li];
    rc = rebuild();
    if (rc) return rc;
    rc = time_classes(cur);
    if (rc) return rc;
    for (int qc = 0; qc < kNumQuartetClasses; ++qc)
      if (cur[qc] < best_ms[qc]) {
        best_ms[qc] = cur[qc];
        best[qc].lane_prims = lp_opts[li];
      }
  }
  for (int qc = 0; qc < kNumQuartetClasses; ++qc) {
    if (best[qc].engine != kEngineReg) {  // the other engines have a fixed launch shape
      best[qc].threads = 128;
      best[qc].persistent = 0;
    }
    cfg[kTuneInts * qc] = best[qc].threads;
    cfg[kTuneInts * qc + 1] = best[qc].lane_prims;
    cfg[kTuneInts * qc + 2] = best[qc].persistent;
    cfg[kTuneInts * qc + 3] = best[qc].engine;
  }
  for (int qc = 0; qc < kNumQuartetClasses; ++qc) c->tune[qc].lane_prims = -1;  // force a rebuild
  rc = jqc_set_tuning(c, cfg);
  if (rc) return rc;
  rc = ensure_jk_tasks(c, precision_mode, mixed_tau, s);
  if (rc) return rc;
  if (cache_path && cache_path[0]) {
    std::FILE* f = std::fopen(cache_path, "a");
    JQC_REQUIRE(f != nullptr, JQC_ERR_INVALID, "jqc_autotune: cannot open the cache file for appending");
    std::fprintf(f, "%s\t", sig.c_str());
    for (int k = 0; k < kTuneInts * kNumQuartetClasses; ++k) std::fprintf(f, k ? " %d" : "%d", cfg[k]);
    std::fprintf(f, "\n");
    std::fclose(f);
  }
  return JQC_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Support for the allocation-free entry point (noalloc.cu).  Runs the J/K
// build of a context whose work list for (precision_mode, mixed_tau) already
// exists, with the per-shell-pair density maxima written to `dmax_scratch`
// (capacity in floats) supplied by the caller.  Never builds a work list and
// never allocates device memory.
namespace jqc {

int ctx_device(const jqc_ctx* c) { return c ? c->device : -1; }

int jk_run_preallocated(jqc_ctx* c, int n_dens, const double* D, double* J, double* K, int precision_mode,
                        double mixed_tau, double dens_tau, float* dmax_scratch, size_t dmax_capacity,
                        cudaStream_t s) {
  JQC_REQUIRE(c && D && J && K && dmax_scratch, JQC_ERR_INVALID, "jqc_jk_noalloc: null argument");
  JQC_REQUIRE(n_dens >= 1 && n_dens <= 4, JQC_ERR_INVALID, "jqc_jk_noalloc: n_dens must be 1..4");
  JQC_REQUIRE(c->pairs_ready, JQC_ERR_NOT_READY, "jqc_jk_noalloc: call jqc_pairs_build first");
  JQC_REQUIRE(precision_mode >= 0 && precision_mode <= 2, JQC_ERR_INVALID, "jqc_jk_noalloc: bad precision_mode");
  JQC_REQUIRE(mixed_tau >= 0.0 && dens_tau >= 0.0, JQC_ERR_INVALID, "jqc_jk_noalloc: thresholds must be >= 0");
  JQC_REQUIRE((size_t)c->n_shell * c->n_shell <= dmax_capacity, JQC_ERR_TOO_LARGE,
              "jqc_jk_noalloc: n_shell^2 exceeds the static scratch (at most 512 shells)");
  const double key_tau = precision_mode == JQC_PREC_MIXED ? mixed_tau : 0.0;
  TaskSet* ts = nullptr;
  for (TaskSet* t : c->jk_cache)
    if (t->valid && t->mode == precision_mode && t->mixed_tau == key_tau) ts = t;
  JQC_REQUIRE(ts != nullptr, JQC_ERR_NOT_READY,
              "jqc_jk_noalloc: no work list for this precision_mode/mixed_tau; call jqc_jk (or jqc_stats) once "
              "with the same settings first, at a point where allocation is allowed");
  int rc = select_device(c);
  if (rc) return rc;
  // the largest block maximum goes after the blocks when the scratch has room
  const size_t nb = (size_t)c->n_shell * c->n_shell;
  float* dmax_top = nb + 1 <= dmax_capacity ? dmax_scratch + nb : nullptr;
  return run_jk_set(c, ts, n_dens, D, J, K, dmax_scratch, dmax_top, dens_tau, s, nullptr);
}

}  // namespace jqc
