// Kernel parameter blocks and launcher declarations shared by the .cu files.
#pragma once

#include "mmd.cuh"

namespace jqc {

constexpr int kNumPairClasses = 6;     // (ss) (ps) (pp) (ds) (dp) (dd)
constexpr int kNumQuartetClasses = 21; // pair class of bra >= ket

__host__ __device__ constexpr int pair_class(int la, int lb) {  // la >= lb
  return la * (la + 1) / 2 + lb;
}
__host__ __device__ constexpr int quartet_class(int pb, int pk) { return pb * (pb + 1) / 2 + pk; }

// Engines that can evaluate a J/K class: the register kernels (lane = ket
// pair, L <= 6), the column engine (compile-time class, lane = ket Cartesian
// pair, L >= 5) and the runtime-class warp engine (every class).
enum JKEngine { kEngineReg = 0, kEngineCol = 1, kEngineWarp = 2 };

struct JKParams {
  const Task* tasks;
  int n_tasks;
  const ShellPair* pairs;
  const void* pp;          // PrimPair* (FP64) or PrimPairF* (FP32)
  const double* centres;   // 3 per shell
  const int* ao;           // first basis function of each shell
  const void* boys;        // Boys table of the kernel's type (row-major)
  const void* boys_al;     // aligned per-order Boys table of the kernel's type
  const double* D;         // n_dens x n x n
  double* J;               // n_dens x n x n (accumulated, symmetrized later)
  double* K;
  int n;
  int n_dens;
  const float* dmax;       // n_shell x n_shell max |D| per shell block, or null
  int n_shell;
  float dens_tau;
  // The largest entry of dmax (one float), or null.  A lane whose bound
  // Q_ab Q_cd 2 max(dmax) is below dens_tau fails the per-block test too, so
  // it leaves before the six block-maximum gathers.
  const float* dmax_top = nullptr;
  int threads = 128;       // threads per block (64, 128, 256)
  int persistent = 0;      // 1: grid capped at the resident blocks, warps stride over tasks
  int engine = kEngineReg; // JKEngine
  // Packed warps (register kernels of bra angular sum <= 2): warp w takes
  // tasks groups[w] .. groups[w+1]-1, at most 32 kets in all, lane by lane.
  // nullptr: one task per warp.
  const int* groups = nullptr;
  int n_groups = 0;
  // Work compacted on the device: warp-sized work item w is items[w] (a
  // group, or a task when there are no groups) for w < *n_items; the
  // register kernels then run a persistent grid, the column and warp engines
  // a grid over the whole list.  nullptr: every item.
  const int* items = nullptr;
  const int* n_items = nullptr;
  // With items: molecule of each shell and the activity flags, so that the
  // lanes of a packed group that hold an inactive molecule's task stay idle.
  const int* shell_mol = nullptr;
  const int* mol_active = nullptr;
};

// One (precision path, class) list for the molecule compaction: its tasks,
// its warp groups (nullptr: one task per item), the item count and where
// the surviving item indices and their count go.
struct CompactSeg {
  const Task* tasks;
  const int* groups;
  int n_items;
  int* out;
  int* count;
  // per item the largest float(Q_bra) * float(Q_ket) of its tasks (the ket
  // runs are Q-descending: their first pair)
  const float* item_q;
};

constexpr int kMaxJKThreads = 256;

struct TensorParams {
  const Task* tasks;
  int n_tasks;
  const ShellPair* pairs;
  const PrimPair* pp;
  const double* centres;
  const int* ao;
  const double* boys;
  const double* boys_al;
  double* eri;
  long long n;
};

struct SchwarzParams {
  const int* pair_ids;     // pairs of one class
  int n_pairs;
  const ShellPair* pairs;
  const PrimPair* pp;
  const double* centres;
  const double* boys;
  const double* boys_al;
  unsigned long long* qmax;  // max (ab|ab) as ordered bits, per pair
};

struct PrimQuartetParams {
  long long n;
  const double* exps;      // 4 per quartet
  const double* centres;   // 12 per quartet
  const double* boys;
  const double* boys_al;
  double* out;             // n x (nab*ncd)
};

// Launchers (return cudaError_t of the launch).
cudaError_t launch_jk(int qc, bool fp32, const JKParams& p, cudaStream_t s);
cudaError_t launch_eri_tensor(int qc, const TensorParams& p, cudaStream_t s);
cudaError_t launch_schwarz(int pc, const SchwarzParams& p, cudaStream_t s);
cudaError_t launch_prim_quartets(int la, int lb, int lc, int ld, const PrimQuartetParams& p, cudaStream_t s);
// tabA: the aligned per-order Boys table of the output type.
cudaError_t launch_boys(const double* T, long long n, int mmax, void* out, bool fp32, const void* tabA, cudaStream_t s);
// dmax[i * n_shell + j] = max |D^s| over the (i, j) shell block and the
// densities; with dmax_top non-null also the largest of them into *dmax_top.
cudaError_t launch_dmax(const double* D, int n_dens, int n, int n_shell, const int* ao, const int* l, float* dmax,
                        float* dmax_top, cudaStream_t s);
cudaError_t launch_symmetrize(double* M, int count, int n, cudaStream_t s);
// Writes, for every segment, the indices of the work items that survive into
// segs[k].out and their count into *segs[k].count (the counts must be zero on
// entry).  An item survives when (with mol_active) one of its tasks belongs to
// an active molecule (mol_active[shell_mol[shell a of the bra pair]] != 0) and
// (with dmax_top) item_q * 2 * (*dmax_top) is not below dens_tau: the class
// kernels' first density test, so every lane of a dropped item would have
// left at that test.  seg_start: n_segs + 1 prefix sums of the item counts.
cudaError_t launch_compact(const CompactSeg* segs, const long long* seg_start, int n_segs, long long total_items,
                           const ShellPair* pairs, const int* shell_mol, const int* mol_active,
                           const float* dmax_top, float dens_tau, cudaStream_t s);

// Class tables: angular momenta of pair class pc.
__host__ __device__ constexpr int pc_la(int pc) { return pc == 0 ? 0 : pc <= 2 ? 1 : 2; }
__host__ __device__ constexpr int pc_lb(int pc) { return pc - pair_class(pc_la(pc), 0); }
__host__ __device__ constexpr int qc_bra(int qc) {
  int pb = 0;
  while ((pb + 1) * (pb + 2) / 2 <= qc) ++pb;
  return pb;
}
__host__ __device__ constexpr int qc_ket(int qc) { return qc - qc_bra(qc) * (qc_bra(qc) + 1) / 2; }
__host__ __device__ constexpr int qc_L(int qc) {
  return pc_la(qc_bra(qc)) + pc_lb(qc_bra(qc)) + pc_la(qc_ket(qc)) + pc_lb(qc_ket(qc));
}
// Classes with L <= 6 run in the register kernels, (dd|dp) and (dd|dd) in the
// warp engine.
__host__ __device__ constexpr bool is_reg_class(int qc) { return qc_L(qc) <= 6; }

struct GradParams {
  const Task* tasks;
  int n_tasks;
  const ShellPair* pairs;
  const PrimPair* pp;
  const double* centres;
  const int* ao;
  const int* atom;        // atom of each shell
  const double* boys;
  const double* boys_al;
  const double* D;        // n_dens x n x n
  int n_dens;
  int n;
  double jscale, kscale;
  double* grad;           // n_atom x 3 (accumulated)
  // Per-shell-pair force slots, 6 per pair (centre a xyz, centre b xyz):
  // the kernels add into these (few collisions) and launch_pair_force_reduce
  // folds them into grad (n_atom x 3 would take every atomic of the launch).
  double* pair_force = nullptr;
  const float* dmax = nullptr;  // n_shell x n_shell max |D^s| per shell block, or null
  const float* dmax_top = nullptr;  // the largest entry of dmax, or null
  int n_shell = 0;
  float dens_tau = 0.f;   // skip quartets whose Gamma bound x Q_ab Q_cd is below this
  int sides = 1;          // register kernels: 2 = bra and ket forces in separate block parts
};

// Gradient engine code of the register kernels with the bra-centre and
// ket-centre forces in separate block parts (GradParams::sides = 2).
constexpr int kGradEngineRegSplit = 3;

// Upper bound of |Gamma_abcd| over a shell quartet from the per-block density
// maxima m (max over the n_dens densities): |D^t| <= n_dens m, so
// |Gamma| <= j n_dens^2 m_ab m_cd + (k/2) n_dens (m_ac m_bd + m_ad m_bc).
__device__ __forceinline__ float gamma_bound(const GradParams& p, int a, int b, int c, int d) {
  const float* m = p.dmax;
  const int ns = p.n_shell;
  const float nd = float(p.n_dens);
  return float(p.jscale) * nd * nd * m[a * ns + b] * m[c * ns + d] +
         0.5f * float(p.kscale) * nd * (m[a * ns + c] * m[b * ns + d] + m[a * ns + d] * m[b * ns + c]);
}

// gamma_bound with every block maximum replaced by their largest, g: the same
// expression tree, so in floating point too it is never below gamma_bound of
// any quartet, and a quartet it screens out is screened out by gamma_bound.
__device__ __forceinline__ float gamma_bound_top(const GradParams& p, float g) {
  const float nd = float(p.n_dens);
  return float(p.jscale) * nd * nd * g * g + 0.5f * float(p.kscale) * nd * (g * g + g * g);
}

struct Grad1Params {
  int n_shell, n, n_atom;
  const int* l;
  const int* nprim;
  const int* prim_off;
  const double* exps;
  const double* coefs;
  const double* centres;
  const int* ao;
  const int* atom;
  const double* atom_xyz;
  const double* atom_Z;
  const int* shell_mol;  // molecule of each shell / atom (nullptr: one molecule)
  const int* atom_mol;
  const double* boys;
  const double* boys_al;  // aligned per-order Boys table
  const double* D;
  const double* W;
  double* grad;
};

// Gradient classes evaluated by the register kernels (L <= 4); the rest use
// the warp-cooperative gradient kernel.
__host__ __device__ constexpr bool is_grad_reg_class(int qc) { return qc_L(qc) <= 4; }
cudaError_t launch_grad_reg(int qc, const GradParams& p, cudaStream_t s);
bool has_grad_row_class(int qc);
cudaError_t launch_grad_row(int qc, const GradParams& p, cudaStream_t s);
cudaError_t launch_warp_grad(int la, int lb, int lc, int ld, const GradParams& p, cudaStream_t s);
cudaError_t launch_grad1e(const Grad1Params& p, cudaStream_t s);
cudaError_t launch_pair_force_reduce(const ShellPair* pairs, int n_pairs, const int* atom, const double* pair_force,
                                     double* grad, cudaStream_t s);

cudaError_t launch_warp_jk(int la, int lb, int lc, int ld, bool fp32, const JKParams& p, cudaStream_t s);
bool has_col_class(int qc);
cudaError_t launch_col_jk(int qc, bool fp32, const JKParams& p, cudaStream_t s);
cudaError_t launch_col_prim(int qc, const PrimQuartetParams& p, cudaStream_t s);  // classes 19, 20

cudaError_t launch_warp_tensor(int la, int lb, int lc, int ld, const TensorParams& p, cudaStream_t s);
cudaError_t launch_warp_schwarz(int la, int lb, const SchwarzParams& p, cudaStream_t s);
cudaError_t launch_warp_prim(int la, int lb, int lc, int ld, const PrimQuartetParams& p, cudaStream_t s);

}  // namespace jqc
