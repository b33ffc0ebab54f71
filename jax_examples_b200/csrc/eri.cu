// ERI-tensor, Schwarz, primitive-quartet and Boys kernels plus small helpers.
#include <algorithm>

#include "jk_impl.cuh"

namespace jqc {

// ----------------------------------------------------------------- Schwarz
// screening.py:32-58: Q_ab = sqrt(max over Cartesian ab of (ab|ab)).
template <int LA, int LB, int NS>
struct SchwarzBody {
  const SchwarzParams& prm;
  int pid;

  template <int PART>
  __device__ __forceinline__ void run() {
    using Cfg = QCfg<LA, LB, LA, LB, NS, PART>;
    if constexpr (Cfg::NCDP > 0) body<PART>();
  }

  template <int PART>
  __device__ __forceinline__ void body() {
    using Cfg = QCfg<LA, LB, LA, LB, NS, PART>;
    const int id = prm.pair_ids[pid];
    const ShellPair bp = prm.pairs[id];
    const double* ctr = prm.centres;
    Vec3<double> A{ctr[3 * bp.a], ctr[3 * bp.a + 1], ctr[3 * bp.a + 2]};
    Vec3<double> B{ctr[3 * bp.b], ctr[3 * bp.b + 1], ctr[3 * bp.b + 2]};
    double out[Cfg::NAB][Cfg::CDP];
    double ebuf[3][LA + 1][LB + 1][LA + LB + 1];
    quartet_accumulate<double, LA, LB, LA, LB, NS, PART, false>(prm.pp + bp.pp, bp.npp, A, B, prm.pp + bp.pp,
                                                                 bp.npp, A, B, prm.boys_al, ebuf, out);
    double m = 0.0;
    static_for<Cfg::NCDP>([&](auto c_) {
      constexpr int cdi = decltype(c_)::value;
      m = fmax(m, out[Cfg::CD0 + cdi][cdi]);
    });
    atomicMax(prm.qmax + id, (unsigned long long)__double_as_longlong(m));
  }
};

template <int LA, int LB>
__global__ void __launch_bounds__(128) schwarz_kernel(const SchwarzParams prm) {
  constexpr int NS = class_split(LA, LB, LA, LB);
  const int pid = blockIdx.x * blockDim.x + threadIdx.x;
  if (pid >= prm.n_pairs) return;
  SchwarzBody<LA, LB, NS> body{prm, pid};
  dispatch_part<NS>(blockIdx.y, body);
}

cudaError_t launch_schwarz(int pc, const SchwarzParams& p, cudaStream_t s) {
  if (p.n_pairs == 0) return cudaSuccess;
  if (!is_reg_class(quartet_class(pc, pc))) return launch_warp_schwarz(pc_la(pc), pc_lb(pc), p, s);
  switch (pc) {
#define S(PC, A, B)                                                       \
  case PC: {                                                              \
    dim3 grid((p.n_pairs + 127) / 128, class_split(A, B, A, B));          \
    schwarz_kernel<A, B><<<grid, 128, 0, s>>>(p);                         \
    return cudaGetLastError();                                            \
  }
    S(0, 0, 0) S(1, 1, 0) S(2, 1, 1) S(3, 2, 0) S(4, 2, 1)
#undef S
    default:
      return cudaErrorInvalidValue;
  }
}

// --------------------------------------------------------- primitive blocks
// obara_saika.py:227-332 primitive_eri_block for a batch of primitive
// quartets with unit coefficients (K_AB and K_CD included).
//
// A block of 128 threads takes kPrimQB = 128 / NS consecutive quartets, one
// thread per (quartet, ket part).  The threads put their part of each block
// into shared memory, and the block's kPrimQB x NAB x NCD outputs, one
// contiguous run of the output array, are stored with consecutive threads on
// consecutive addresses: a thread storing its own block element by element
// would touch one cache line per lane in every store instruction.
template <int NS>
constexpr int prim_qb() { return NS >= 128 ? 1 : 128 / NS; }

template <int LA, int LB, int LC, int LD, int NS>
struct PrimBody {
  const PrimQuartetParams& prm;
  long long q;
  double* blk;  // this quartet's NAB x NCD block in shared memory

  template <int PART>
  __device__ __forceinline__ void run() {
    using Cfg = QCfg<LA, LB, LC, LD, NS, PART>;
    if constexpr (Cfg::NCDP > 0) body<PART>();
  }

  template <int PART>
  __device__ __forceinline__ void body() {
    using Cfg = QCfg<LA, LB, LC, LD, NS, PART>;
    const double* ex = prm.exps + 4 * q;
    const double* c = prm.centres + 12 * q;
    Vec3<double> A{c[0], c[1], c[2]}, B{c[3], c[4], c[5]}, C{c[6], c[7], c[8]}, D{c[9], c[10], c[11]};
    PrimPair bra, ket;
    {
      const double al = ex[0], be = ex[1], p = al + be;
      const double dx = A.x - B.x, dy = A.y - B.y, dz = A.z - B.z;
      bra = PrimPair{p, 0.5 / p, (al * A.x + be * B.x) / p, (al * A.y + be * B.y) / p, (al * A.z + be * B.z) / p,
                     exp(-(al * be / p) * (dx * dx + dy * dy + dz * dz)), al, be};
    }
    {
      const double al = ex[2], be = ex[3], p = al + be;
      const double dx = C.x - D.x, dy = C.y - D.y, dz = C.z - D.z;
      ket = PrimPair{p, 0.5 / p, (al * C.x + be * D.x) / p, (al * C.y + be * D.y) / p, (al * C.z + be * D.z) / p,
                     exp(-(al * be / p) * (dx * dx + dy * dy + dz * dz)), al, be};
    }
    double out[Cfg::NAB][Cfg::CDP];
    double ebuf[3][LA + 1][LB + 1][LA + LB + 1];
    quartet_accumulate<double, LA, LB, LC, LD, NS, PART, false, false>(&bra, 1, A, B, &ket, 1, C, D, prm.boys_al,
                                                                        ebuf, out);
    static_for<Cfg::NAB * Cfg::NCDP>([&](auto x_) {
      constexpr int x = decltype(x_)::value;
      constexpr int ab = x / Cfg::NCDP, cdi = x % Cfg::NCDP;
      blk[ab * Cfg::NCD + Cfg::CD0 + cdi] = out[ab][cdi];
    });
  }
};

template <int LA, int LB, int LC, int LD>
__global__ void __launch_bounds__(128) prim_kernel(const PrimQuartetParams prm) {
  constexpr int NS = class_split(LA, LB, LC, LD);
  constexpr int QB = prim_qb<NS>();
  constexpr int NE = ncart(LA) * ncart(LB) * ncart(LC) * ncart(LD);
  __shared__ double s_out[QB * NE];
  const long long q0 = (long long)blockIdx.x * QB;
  const int nq = (int)(prm.n - q0 < QB ? prm.n - q0 : QB);
  const int ql = int(threadIdx.x) % QB, part = int(threadIdx.x) / QB;
  if (ql < nq && part < NS) {
    PrimBody<LA, LB, LC, LD, NS> body{prm, q0 + ql, s_out + ql * NE};
    dispatch_part<NS>(part, body);
  }
  __syncthreads();
  double* o = prm.out + q0 * NE;
  for (int i = int(threadIdx.x); i < nq * NE; i += int(blockDim.x)) o[i] = s_out[i];
}

cudaError_t launch_prim_quartets(int la, int lb, int lc, int ld, const PrimQuartetParams& p, cudaStream_t s) {
  if (p.n == 0) return cudaSuccess;
  if (la < lb || lc < ld || la > 2 || lc > 2) return cudaErrorInvalidValue;
  const int pb = pair_class(la, lb), pk = pair_class(lc, ld);
  if (pb < pk) return cudaErrorInvalidValue;
  if (!is_reg_class(quartet_class(pb, pk))) return launch_col_prim(quartet_class(pb, pk), p, s);
  switch (quartet_class(pb, pk)) {
#define X(Q, A, B, C, D)                                                                     \
  case Q: {                                                                                  \
    constexpr long long qb = prim_qb<class_split(A, B, C, D)>();                            \
    prim_kernel<A, B, C, D><<<(unsigned)((p.n + qb - 1) / qb), 128, 0, s>>>(p);              \
    return cudaGetLastError();                                                               \
  }
    JQC_FOR_REG_CLASSES(X)
#undef X
    default:
      return cudaErrorInvalidValue;
  }
}

// -------------------------------------------------------------------- Boys
// One thread per argument, the order fixed at compile time (the aligned
// per-order table and an unrolled recursion); the block's outputs are staged
// in shared memory and written back as one contiguous, coalesced run.
template <typename T, int M>
__global__ void __launch_bounds__(256) boys_kernel(const double* __restrict__ tv, long long n, T* __restrict__ out,
                                                   const T* __restrict__ tabA) {
  __shared__ T stage[256 * (M + 1)];
  const long long base = (long long)blockIdx.x * 256;
  const long long i = base + threadIdx.x;
  if (i < n) {
    const double t = tv[i];
    T F[M + 1];
    if (t >= 0.0) {
      boys_eval<T, M>(T(t), tabA, F);
    } else {  // negative or NaN argument: no table access
#pragma unroll
      for (int m = 0; m <= M; ++m) F[m] = T(NAN);
    }
#pragma unroll
    for (int m = 0; m <= M; ++m) stage[threadIdx.x * (M + 1) + m] = F[m];
  }
  __syncthreads();
  const long long cnt = (n - base < 256 ? n - base : 256) * (M + 1);
  T* dst = out + base * (M + 1);
  for (long long k = threadIdx.x; k < cnt; k += 256) dst[k] = stage[k];
}

template <typename T>
static cudaError_t launch_boys_t(const double* tv, long long n, int mmax, T* out, const T* tabA, cudaStream_t s) {
  const unsigned g = (unsigned)((n + 255) / 256);
  switch (mmax) {
#define B(Mv)                                                   \
  case Mv:                                                      \
    boys_kernel<T, Mv><<<g, 256, 0, s>>>(tv, n, out, tabA);     \
    break;
    B(0) B(1) B(2) B(3) B(4) B(5) B(6) B(7) B(8) B(9) B(10) B(11) B(12) B(13) B(14) B(15) B(16)
#undef B
    default:
      return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_boys(const double* T, long long n, int mmax, void* out, bool fp32, const void* tabA,
                        cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  if (fp32) return launch_boys_t<float>(T, n, mmax, static_cast<float*>(out), static_cast<const float*>(tabA), s);
  return launch_boys_t<double>(T, n, mmax, static_cast<double*>(out), static_cast<const double*>(tabA), s);
}

// --------------------------------------------------------------- helpers
__global__ void dmax_kernel(const double* __restrict__ D, int n_dens, int n, int n_shell, const int* __restrict__ ao,
                            const int* __restrict__ l, float* __restrict__ dmax, float* __restrict__ dmax_top) {
  const long long tot = (long long)n_shell * n_shell;
  float top = 0.f;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < tot;
       idx += (long long)gridDim.x * blockDim.x) {
    const int i = int(idx / n_shell), j = int(idx % n_shell);
    const int ni = ncart(l[i]), nj = ncart(l[j]);
    double m = 0.0;
    for (int d = 0; d < n_dens; ++d)
      for (int a = 0; a < ni; ++a)
        for (int b = 0; b < nj; ++b) m = fmax(m, fabs(D[(size_t)d * n * n + (size_t)(ao[i] + a) * n + ao[j] + b]));
    dmax[idx] = float(m);
    top = fmaxf(top, float(m));
  }
  if (dmax_top == nullptr) return;  // uniform over the launch
  // block maximum, then one atomic per block: non-negative floats order as
  // their bit patterns do
  __shared__ float warp_top[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) top = fmaxf(top, __shfl_xor_sync(0xffffffffu, top, o));
  if ((threadIdx.x & 31) == 0) warp_top[threadIdx.x >> 5] = top;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    for (int w = 0; w < int(blockDim.x >> 5); ++w) t = fmaxf(t, warp_top[w]);
    if (t > 0.f) atomicMax(reinterpret_cast<int*>(dmax_top), __float_as_int(t));
  }
}

cudaError_t launch_dmax(const double* D, int n_dens, int n, int n_shell, const int* ao, const int* l, float* dmax,
                        float* dmax_top, cudaStream_t s) {
  const long long tot = (long long)n_shell * n_shell;
  if (dmax_top != nullptr) {
    const cudaError_t e = cudaMemsetAsync(dmax_top, 0, sizeof(float), s);
    if (e != cudaSuccess) return e;
  }
  if (tot == 0) return cudaSuccess;
  const long long blocks = std::min<long long>((tot + 255) / 256, 2048);
  dmax_kernel<<<(unsigned)blocks, 256, 0, s>>>(D, n_dens, n, n_shell, ao, l, dmax, dmax_top);
  return cudaGetLastError();
}

// Molecule compaction of the work items of many lists at once: thread g takes
// item g of the concatenated lists (segment by binary search on the prefix
// sums), keeps it when one of its tasks belongs to an active molecule, and
// the lanes of a warp that keep items of the same segment append them with
// one atomic.  The order inside a segment follows the warps' progress.
__global__ void __launch_bounds__(256) compact_kernel(const CompactSeg* __restrict__ segs,
                                                      const long long* __restrict__ seg_start, int n_segs,
                                                      long long total, const ShellPair* __restrict__ pairs,
                                                      const int* __restrict__ shell_mol,
                                                      const int* __restrict__ mol_active,
                                                      const float* __restrict__ dmax_top, float dens_tau) {
  // 2 x the largest density block maximum: the kernels' bound, same operands
  const float top2 = dmax_top != nullptr ? 2.f * *dmax_top : 0.f;
  const int lane = threadIdx.x & 31;
  const long long step = (long long)gridDim.x * blockDim.x;
  for (long long base = (long long)blockIdx.x * blockDim.x; base < total; base += step) {
    const long long g = base + threadIdx.x;
    int seg = -1, item = 0;
    bool act = false;
    if (g < total) {
      int lo = 0, hi = n_segs - 1;  // last segment starting at or before g
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (seg_start[mid] <= g)
          lo = mid;
        else
          hi = mid - 1;
      }
      seg = lo;
      item = int(g - seg_start[seg]);
      const CompactSeg S = segs[seg];
      act = true;
      if (dmax_top != nullptr) act = !(S.item_q[item] * top2 < dens_tau);
      if (act && mol_active != nullptr) {
        act = false;
        if (S.groups != nullptr) {
          for (int t = S.groups[item]; t < S.groups[item + 1] && !act; ++t)
            act = mol_active[shell_mol[pairs[S.tasks[t].bra].a]] != 0;
        } else {
          act = mol_active[shell_mol[pairs[S.tasks[item].bra].a]] != 0;
        }
      }
    }
    const unsigned same = __match_any_sync(0xffffffffu, act ? seg : -1);
    if (act) {
      const int leader = __ffs(same) - 1;
      const int rank = __popc(same & ((1u << lane) - 1u));
      int slot = 0;
      if (lane == leader) slot = atomicAdd(segs[seg].count, __popc(same));
      slot = __shfl_sync(same, slot, leader);
      segs[seg].out[slot + rank] = item;
    }
  }
}

cudaError_t launch_compact(const CompactSeg* segs, const long long* seg_start, int n_segs, long long total_items,
                           const ShellPair* pairs, const int* shell_mol, const int* mol_active,
                           const float* dmax_top, float dens_tau, cudaStream_t s) {
  if (total_items == 0 || n_segs == 0) return cudaSuccess;
  int dev = 0, sms = 148;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  const long long want = (total_items + 255) / 256;
  const int blocks = (int)std::min<long long>(want, (long long)sms * 8);
  compact_kernel<<<blocks, 256, 0, s>>>(segs, seg_start, n_segs, total_items, pairs, shell_mol, mol_active,
                                        dmax_top, dens_tau);
  return cudaGetLastError();
}

// M <- M + M^T for `count` consecutive n x n matrices.
__global__ void symmetrize_kernel(double* M, int count, int n) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nn = (long long)n * n;
  if (idx >= nn * count) return;
  const int m = int(idx / nn);
  const int i = int((idx % nn) / n), j = int(idx % n);
  if (i < j) return;
  double* A = M + m * nn;
  if (i == j) {
    A[(size_t)i * n + i] *= 2.0;
  } else {
    const double v = A[(size_t)i * n + j] + A[(size_t)j * n + i];
    A[(size_t)i * n + j] = v;
    A[(size_t)j * n + i] = v;
  }
}

cudaError_t launch_symmetrize(double* M, int count, int n, cudaStream_t s) {
  const long long tot = (long long)n * n * count;
  if (tot == 0) return cudaSuccess;
  symmetrize_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(M, count, n);
  return cudaGetLastError();
}

}  // namespace jqc
