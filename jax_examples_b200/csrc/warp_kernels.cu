// Kernels of the warp-cooperative engine (classes with L >= 5).
#include "warp_engine.cuh"

namespace jqc {

constexpr int kWarpBlock = 128;  // 4 warps per block

template <typename T>
__device__ __forceinline__ WarpSmem<T>* warp_smem() {
  extern __shared__ __align__(16) unsigned char smraw[];
  return reinterpret_cast<WarpSmem<T>*>(smraw) + (threadIdx.x >> 5);
}

template <typename T>
__device__ __forceinline__ void warp_contract_pair(WarpQuartet<T>& wq, const typename PPType<T>::type* bra, int nbra,
                                                   Vec3<T> A, Vec3<T> B, const typename PPType<T>::type* ket,
                                                   int nket, Vec3<T> C, Vec3<T> D, const T* tab) {
  for (int ip = 0; ip < nbra; ++ip) {
    const auto bp = bra[ip];
    wq.set_bra(T(bp.Px), T(bp.Py), T(bp.Pz), T(bp.h), A, B);
    for (int iq = 0; iq < nket; ++iq) {
      const auto kp = ket[iq];
      wq.add_prim(T(bp.p), T(bp.h), T(bp.Px), T(bp.Py), T(bp.Pz), T(bp.K), T(kp.p), T(kp.h), T(kp.Px), T(kp.Py),
                  T(kp.Pz), T(kp.K), C, D, tab);
    }
  }
  wq.publish();
}

template <typename T>
__device__ __forceinline__ Vec3<T> centre(const double* c, int s) {
  return Vec3<T>{T(c[3 * s]), T(c[3 * s + 1]), T(c[3 * s + 2])};
}

// ------------------------------------------------------------------ J/K
template <typename T>
__global__ void __launch_bounds__(kWarpBlock) warp_jk_kernel(const JKParams prm, int la, int lb, int lc, int ld) {
  using PPT = typename PPType<T>::type;
  WarpSmem<T>* sm = warp_smem<T>();
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= prm.n_tasks) return;
  if (prm.items != nullptr) {  // compacted work: the grid covers the whole list
    if (warp >= *prm.n_items) return;
    warp = prm.items[warp];
  }
  const Task task = prm.tasks[warp];
  const ShellPair bp = prm.pairs[task.bra];
  const PPT* pp = static_cast<const PPT*>(prm.pp);
  const T* tab = static_cast<const T*>(prm.boys);
  const int na = ncart(la), nb = ncart(lb), nc = ncart(lc), nd = ncart(ld);
  const int n = prm.n;
  WarpQuartet<T> wq;
  wq.sm = sm;
  wq.lane = lane;
  for (int kk = 0; kk < task.nket; ++kk) {
    const int kidx = task.ket0 + kk;
    const ShellPair kp = prm.pairs[kidx];
    if (prm.dmax_top != nullptr && float(bp.Q) * float(kp.Q) * (2.f * *prm.dmax_top) < prm.dens_tau)
      continue;  // below the bound for any density block
    if (prm.dmax != nullptr) {
      const float* dm = prm.dmax;
      const int ns = prm.n_shell;
      float m = fmaxf(2.f * dm[bp.a * ns + bp.b], 2.f * dm[kp.a * ns + kp.b]);
      m = fmaxf(m, fmaxf(dm[bp.a * ns + kp.a], dm[bp.a * ns + kp.b]));
      m = fmaxf(m, fmaxf(dm[bp.b * ns + kp.a], dm[bp.b * ns + kp.b]));
      if (float(bp.Q) * float(kp.Q) * m < prm.dens_tau) continue;  // uniform over the warp
    }
    wq.init(la, lb, lc, ld);
    const int p0 = task.flags & 0xffff, p1 = task.flags >> 16;
    warp_contract_pair<T>(wq, pp + bp.pp + p0, p1 - p0, centre<T>(prm.centres, bp.a), centre<T>(prm.centres, bp.b),
                          pp + kp.pp, kp.npp, centre<T>(prm.centres, kp.a), centre<T>(prm.centres, kp.b), tab);
    double s = 1.0;
    if (bp.diag) s *= 0.5;
    if (kp.diag) s *= 0.5;
    if (task.bra == kidx) s *= 0.5;
    warp_digest_jk<T>(prm, sm->XB, na, nb, nc, nd, prm.ao[bp.a], prm.ao[bp.b], prm.ao[kp.a], prm.ao[kp.b], s, lane);
    __syncwarp();
  }
}

// --------------------------------------------------------------- tensor
__global__ void __launch_bounds__(kWarpBlock) warp_tensor_kernel(const TensorParams prm, int la, int lb, int lc,
                                                                 int ld) {
  WarpSmem<double>* sm = warp_smem<double>();
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= prm.n_tasks) return;
  const Task task = prm.tasks[warp];
  const ShellPair bp = prm.pairs[task.bra];
  const int nb = ncart(lb), nc = ncart(lc), nd = ncart(ld);
  const long long n = prm.n;
  WarpQuartet<double> wq;
  wq.sm = sm;
  wq.lane = lane;
  for (int kk = 0; kk < task.nket; ++kk) {
    const ShellPair kp = prm.pairs[task.ket0 + kk];
    wq.init(la, lb, lc, ld);
    warp_contract_pair<double>(wq, prm.pp + bp.pp, bp.npp, centre<double>(prm.centres, bp.a),
                               centre<double>(prm.centres, bp.b), prm.pp + kp.pp, kp.npp,
                               centre<double>(prm.centres, kp.a), centre<double>(prm.centres, kp.b), prm.boys);
    const long long a0 = prm.ao[bp.a], b0 = prm.ao[bp.b], c0 = prm.ao[kp.a], d0 = prm.ao[kp.b];
    const int ncd = nc * nd;
    double* e = prm.eri;
    for (int x = lane; x < wq.ntot; x += 32) {
      const int ab = x / ncd, cd = x % ncd;
      const long long i = a0 + ab / nb, j = b0 + ab % nb, k = c0 + cd / nd, l = d0 + cd % nd;
      const double v = sm->XB[x];
      e[((i * n + j) * n + k) * n + l] = v;
      e[((j * n + i) * n + k) * n + l] = v;
      e[((i * n + j) * n + l) * n + k] = v;
      e[((j * n + i) * n + l) * n + k] = v;
      e[((k * n + l) * n + i) * n + j] = v;
      e[((l * n + k) * n + i) * n + j] = v;
      e[((k * n + l) * n + j) * n + i] = v;
      e[((l * n + k) * n + j) * n + i] = v;
    }
    __syncwarp();
  }
}

// -------------------------------------------------------------- Schwarz
__global__ void __launch_bounds__(kWarpBlock) warp_schwarz_kernel(const SchwarzParams prm, int la, int lb) {
  WarpSmem<double>* sm = warp_smem<double>();
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= prm.n_pairs) return;
  const int id = prm.pair_ids[warp];
  const ShellPair bp = prm.pairs[id];
  WarpQuartet<double> wq;
  wq.sm = sm;
  wq.lane = lane;
  wq.init(la, lb, la, lb);
  const Vec3<double> A = centre<double>(prm.centres, bp.a), B = centre<double>(prm.centres, bp.b);
  warp_contract_pair<double>(wq, prm.pp + bp.pp, bp.npp, A, B, prm.pp + bp.pp, bp.npp, A, B, prm.boys);
  const int nab = ncart(la) * ncart(lb);
  double m = 0.0;
  for (int ab = lane; ab < nab; ab += 32) m = fmax(m, sm->XB[ab * nab + ab]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if (lane == 0) atomicMax(prm.qmax + id, (unsigned long long)__double_as_longlong(m));
}

// ------------------------------------------------------- primitive blocks
__global__ void __launch_bounds__(kWarpBlock) warp_prim_kernel(const PrimQuartetParams prm, int la, int lb, int lc,
                                                               int ld) {
  WarpSmem<double>* sm = warp_smem<double>();
  const long long q = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (q >= prm.n) return;
  const double* ex = prm.exps + 4 * q;
  const double* c = prm.centres + 12 * q;
  const Vec3<double> A{c[0], c[1], c[2]}, B{c[3], c[4], c[5]}, C{c[6], c[7], c[8]}, D{c[9], c[10], c[11]};
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
  WarpQuartet<double> wq;
  wq.sm = sm;
  wq.lane = lane;
  wq.init(la, lb, lc, ld);
  warp_contract_pair<double>(wq, &bra, 1, A, B, &ket, 1, C, D, prm.boys);
  double* o = prm.out + q * wq.ntot;
  for (int x = lane; x < wq.ntot; x += 32) o[x] = sm->XB[x];
}

// ------------------------------------------------------------- launchers
template <typename K>
static cudaError_t set_smem(K kernel, size_t bytes) {
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

cudaError_t launch_warp_jk(int la, int lb, int lc, int ld, bool fp32, const JKParams& p, cudaStream_t s) {
  if (p.n_tasks == 0) return cudaSuccess;
  const unsigned grid = (unsigned)((p.n_tasks + 3) / 4);
  if (fp32) {
    const size_t sm = 4 * sizeof(WarpSmem<float>);
    cudaError_t e = set_smem(warp_jk_kernel<float>, sm);
    if (e != cudaSuccess) return e;
    warp_jk_kernel<float><<<grid, kWarpBlock, sm, s>>>(p, la, lb, lc, ld);
  } else {
    const size_t sm = 4 * sizeof(WarpSmem<double>);
    cudaError_t e = set_smem(warp_jk_kernel<double>, sm);
    if (e != cudaSuccess) return e;
    warp_jk_kernel<double><<<grid, kWarpBlock, sm, s>>>(p, la, lb, lc, ld);
  }
  return cudaGetLastError();
}

cudaError_t launch_warp_tensor(int la, int lb, int lc, int ld, const TensorParams& p, cudaStream_t s) {
  if (p.n_tasks == 0) return cudaSuccess;
  const size_t sm = 4 * sizeof(WarpSmem<double>);
  cudaError_t e = set_smem(warp_tensor_kernel, sm);
  if (e != cudaSuccess) return e;
  warp_tensor_kernel<<<(unsigned)((p.n_tasks + 3) / 4), kWarpBlock, sm, s>>>(p, la, lb, lc, ld);
  return cudaGetLastError();
}

cudaError_t launch_warp_schwarz(int la, int lb, const SchwarzParams& p, cudaStream_t s) {
  if (p.n_pairs == 0) return cudaSuccess;
  const size_t sm = 4 * sizeof(WarpSmem<double>);
  cudaError_t e = set_smem(warp_schwarz_kernel, sm);
  if (e != cudaSuccess) return e;
  warp_schwarz_kernel<<<(unsigned)((p.n_pairs + 3) / 4), kWarpBlock, sm, s>>>(p, la, lb);
  return cudaGetLastError();
}

cudaError_t launch_warp_prim(int la, int lb, int lc, int ld, const PrimQuartetParams& p, cudaStream_t s) {
  if (p.n == 0) return cudaSuccess;
  const size_t sm = 4 * sizeof(WarpSmem<double>);
  cudaError_t e = set_smem(warp_prim_kernel, sm);
  if (e != cudaSuccess) return e;
  warp_prim_kernel<<<(unsigned)((p.n + 3) / 4), kWarpBlock, sm, s>>>(p, la, lb, lc, ld);
  return cudaGetLastError();
}

}  // namespace jqc
