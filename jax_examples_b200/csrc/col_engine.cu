// Column engine for the high angular-momentum J/K classes (L >= 5).
//
// One warp evaluates one contracted shell quartet (ab|cd) of a class fixed at
// compile time; lane c owns the ket Cartesian pair cd = c (and c + 32 when a
// class has more than 32).  Per primitive quartet:
//   * lanes 0..2 build the bra E coefficients of one axis each (once per bra
//     primitive pair), lanes 3..5 the ket E (with (-1)^t), lanes 0..L the
//     Boys values F_m(T) times the prefactor, all into the warp's slice of
//     shared memory; the R_tuv recursion then runs in shared memory, lanes
//     parallel over the entries of one total order;
//   * each lane contracts its ket pair: G[h'] = F^x F^y F^z over the ket
//     Hermite index h' (zero beyond c+d, so the loops are compile-time),
//     X[h] = sum_h' G[h'] R[h + h'] for every bra Hermite index h (R read at
//     the same address by all lanes: a broadcast), and
//     block[ab][cd] += sum_tuv E^x E^y E^z X_tuv with the bra E read by all
//     lanes at the same address.
// Unlike the register kernels (lane = ket pair, the whole class per thread)
// no thread holds more than the two Hermite vectors G and X, and unlike the
// runtime-class warp engine every index is a compile-time constant.
// Digestion into J/K is the warp engine's (warp_digest_jk).
#include "warp_engine.cuh"

namespace jqc {

__host__ __device__ constexpr int herm_order(int h) {
  int s = 0;
  while (nherm(s) <= h) ++s;
  return s;
}
__host__ __device__ constexpr int herm_t(int h) {
  const int s = herm_order(h);
  return cart_lx(s, h - nherm(s - 1));
}
__host__ __device__ constexpr int herm_u(int h) {
  const int s = herm_order(h);
  return cart_ly(s, h - nherm(s - 1));
}
__host__ __device__ constexpr int herm_v(int h) { return herm_order(h) - herm_t(h) - herm_u(h); }

template <typename T, int LA, int LB, int LC, int LD>
struct ColSmem {
  static constexpr int LAB = LA + LB, LCD = LC + LD, L = LAB + LCD;
  static constexpr int NAB = ncart(LA) * ncart(LB), NCD = ncart(LC) * ncart(LD);
  T Eb[3][LA + 1][LB + 1][LAB + 1];
  T Fk[3][LC + 1][LD + 1][LCD + 1];  // zero beyond t = c + d
  T R[nherm(L)];
  T Rn[L + 1];
  T blk[NAB * NCD];
};

constexpr int kColWarps = 4;

// Bra E coefficients of one bra primitive pair (lanes 0..2, one axis each).
// The caller synchronises the warp before (earlier readers) and after.
template <typename T, int LA, int LB, int LC, int LD>
__device__ __forceinline__ void col_set_bra(ColSmem<T, LA, LB, LC, LD>* sm, const typename PPType<T>::type& bp,
                                            Vec3<T> A, Vec3<T> B, int lane) {
  if (lane == 0) ecoef_compute<T, LA, LB, false>(sm->Eb[0], bp.Px - A.x, bp.Px - B.x, bp.h);
  if (lane == 1) ecoef_compute<T, LA, LB, false>(sm->Eb[1], bp.Py - A.y, bp.Py - B.y, bp.h);
  if (lane == 2) ecoef_compute<T, LA, LB, false>(sm->Eb[2], bp.Pz - A.z, bp.Pz - B.z, bp.h);
}

// Adds one primitive quartet (bra E already in sm->Eb) to sm->blk; all
// lanes call with the same arguments and leave the warp synchronised.
template <typename T, int LA, int LB, int LC, int LD>
__device__ __forceinline__ void col_add_prim(ColSmem<T, LA, LB, LC, LD>* sm, const typename PPType<T>::type& bp,
                                             const typename PPType<T>::type& kp, Vec3<T> C, Vec3<T> D,
                                             const T* __restrict__ tab, int lane) {
  using S = ColSmem<T, LA, LB, LC, LD>;
  constexpr int L = S::L, LAB = S::LAB, LCD = S::LCD, NCD = S::NCD;
  constexpr int NA = ncart(LA), NB = ncart(LB), ND = ncart(LD);
  if (lane == 3) ecoef_compute<T, LC, LD, true>(sm->Fk[0], kp.Px - C.x, kp.Px - D.x, kp.h);
  if (lane == 4) ecoef_compute<T, LC, LD, true>(sm->Fk[1], kp.Py - C.y, kp.Py - D.y, kp.h);
  if (lane == 5) ecoef_compute<T, LC, LD, true>(sm->Fk[2], kp.Pz - C.z, kp.Pz - D.z, kp.h);
  const T r = fast_rsqrt(bp.p + kp.p);
  const T rho = bp.p * kp.p * (r * r);
  const T X = bp.Px - kp.Px, Y = bp.Py - kp.Py, Z = bp.Pz - kp.Pz;
  const T tb = rho * (X * X + Y * Y + Z * Z);
  if (lane <= L) {
    T pref = T(4.0 * kTwoPi25) * bp.K * kp.K * (bp.h * kp.h) * r;
    const T m2rho = T(-2) * rho;
    for (int k = 0; k < lane; ++k) pref *= m2rho;
    sm->Rn[lane] = pref * boys_single<T>(tb, lane, tab);
  }
  __syncwarp();
  warp_hermite_R<T, L>(sm->R, sm->Rn, X, Y, Z, lane);
  for (int c = lane; c < NCD; c += 32) {
    const int ci = c / ND, di = c - (c / ND) * ND;
    const int cx = cart_lx(LC, ci), cy = cart_ly(LC, ci), cz = LC - cx - cy;
    const int dx = cart_lx(LD, di), dy = cart_ly(LD, di), dz = LD - dx - dy;
    T G[nherm(LCD)];
    static_for<nherm(LCD)>([&](auto h_) {
      constexpr int h = decltype(h_)::value;
      constexpr int ht = herm_t(h), hu = herm_u(h), hv = herm_v(h);
      G[h] = sm->Fk[0][cx][dx][ht] * sm->Fk[1][cy][dy][hu] * sm->Fk[2][cz][dz][hv];
    });
    T Xh[nherm(LAB)];
    static_for<nherm(LAB)>([&](auto h_) {
      constexpr int h = decltype(h_)::value;
      constexpr int ht = herm_t(h), hu = herm_u(h), hv = herm_v(h);
      T x = T(0);
      static_for<nherm(LCD)>([&](auto g_) {
        constexpr int g = decltype(g_)::value;
        constexpr int ri = herm_index(ht + herm_t(g), hu + herm_u(g), hv + herm_v(g));
        x += G[g] * sm->R[ri];
      });
      Xh[h] = x;
    });
    static_for<NA>([&](auto a_) {
      constexpr int a = decltype(a_)::value;
      constexpr int ax = cart_lx(LA, a), ay = cart_ly(LA, a), az = cart_lz(LA, a);
      static_for<NB>([&](auto b_) {
        constexpr int b = decltype(b_)::value;
        constexpr int bx = cart_lx(LB, b), by = cart_ly(LB, b), bz = cart_lz(LB, b);
        T acc = T(0);
        static_for<ax + bx + 1>([&](auto t_) {
          constexpr int t = decltype(t_)::value;
          static_for<ay + by + 1>([&](auto u_) {
            constexpr int u = decltype(u_)::value;
            const T exy = sm->Eb[0][ax][bx][t] * sm->Eb[1][ay][by][u];
            static_for<az + bz + 1>([&](auto v_) {
              constexpr int v = decltype(v_)::value;
              acc += exy * sm->Eb[2][az][bz][v] * Xh[herm_index(t, u, v)];
            });
          });
        });
        sm->blk[(a * NB + b) * NCD + c] += acc;
      });
    });
  }
  __syncwarp();
}

// Accumulates block[ab][cd] of one shell quartet over bra primitive pairs
// [0, nbra) and ket primitive pairs [0, nket) into sm->blk (zeroed here).
template <typename T, int LA, int LB, int LC, int LD>
__device__ __forceinline__ void col_quartet(ColSmem<T, LA, LB, LC, LD>* sm, const typename PPType<T>::type* bra,
                                            int nbra, Vec3<T> A, Vec3<T> B, const typename PPType<T>::type* ket,
                                            int nket, Vec3<T> C, Vec3<T> D, const T* __restrict__ tab, int lane) {
  using S = ColSmem<T, LA, LB, LC, LD>;
  using PPT = typename PPType<T>::type;
  for (int i = lane; i < S::NAB * S::NCD; i += 32) sm->blk[i] = T(0);
  for (int ip = 0; ip < nbra; ++ip) {
    const PPT bp = ld_pp(bra + ip);
    __syncwarp();
    col_set_bra<T, LA, LB, LC, LD>(sm, bp, A, B, lane);
    for (int iq = 0; iq < nket; ++iq) {
      const PPT kp = ld_pp(ket + iq);
      col_add_prim<T, LA, LB, LC, LD>(sm, bp, kp, C, D, tab, lane);
    }
  }
  __syncwarp();
}

template <typename T, int LA, int LB, int LC, int LD>
__global__ void __launch_bounds__(32 * kColWarps) col_jk_kernel(const JKParams prm) {
  using S = ColSmem<T, LA, LB, LC, LD>;
  using PPT = typename PPType<T>::type;
  extern __shared__ __align__(16) unsigned char col_smraw[];
  S* sm = reinterpret_cast<S*>(col_smraw) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (warp >= prm.n_tasks) return;
  if (prm.items != nullptr) {  // compacted work: the grid covers the whole list
    if (warp >= *prm.n_items) return;
    warp = prm.items[warp];
  }
  // E entries beyond t = i + j are never written by ecoef_compute: zero them once
  for (int i = lane; i < int(sizeof(sm->Fk) / sizeof(T)); i += 32) (&sm->Fk[0][0][0][0])[i] = T(0);
  for (int i = lane; i < int(sizeof(sm->Eb) / sizeof(T)); i += 32) (&sm->Eb[0][0][0][0])[i] = T(0);
  __syncwarp();
  const Task task = prm.tasks[warp];
  const ShellPair bp = prm.pairs[task.bra];
  const PPT* pp = static_cast<const PPT*>(prm.pp);
  const T* tab = static_cast<const T*>(prm.boys);
  const double* ctr = prm.centres;
  const Vec3<T> A{T(ctr[3 * bp.a]), T(ctr[3 * bp.a + 1]), T(ctr[3 * bp.a + 2])};
  const Vec3<T> B{T(ctr[3 * bp.b]), T(ctr[3 * bp.b + 1]), T(ctr[3 * bp.b + 2])};
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
    const Vec3<T> C{T(ctr[3 * kp.a]), T(ctr[3 * kp.a + 1]), T(ctr[3 * kp.a + 2])};
    const Vec3<T> Dv{T(ctr[3 * kp.b]), T(ctr[3 * kp.b + 1]), T(ctr[3 * kp.b + 2])};
    const int p0 = task.flags & 0xffff, p1 = task.flags >> 16;
    col_quartet<T, LA, LB, LC, LD>(sm, pp + bp.pp + p0, p1 - p0, A, B, pp + kp.pp, kp.npp, C, Dv, tab, lane);
    double s = 1.0;
    if (bp.diag) s *= 0.5;
    if (kp.diag) s *= 0.5;
    if (task.bra == kidx) s *= 0.5;
    warp_digest_jk<T>(prm, sm->blk, ncart(LA), ncart(LB), ncart(LC), ncart(LD), prm.ao[bp.a], prm.ao[bp.b],
                      prm.ao[kp.a], prm.ao[kp.b], s, lane);
    __syncwarp();
  }
}

template <typename T, int LA, int LB, int LC, int LD>
static cudaError_t launch_col_jk_class(const JKParams& p, cudaStream_t s) {
  if (p.n_tasks == 0) return cudaSuccess;
  const size_t sm = kColWarps * sizeof(ColSmem<T, LA, LB, LC, LD>);
  static bool configured = false;
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(col_jk_kernel<T, LA, LB, LC, LD>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    configured = true;
  }
  const unsigned grid = (unsigned)((p.n_tasks + kColWarps - 1) / kColWarps);
  col_jk_kernel<T, LA, LB, LC, LD><<<grid, 32 * kColWarps, sm, s>>>(p);
  return cudaGetLastError();
}

// Primitive blocks (obara_saika.py:227-332 primitive_eri_block with unit
// coefficients, K_AB and K_CD included) of the high-L classes: one warp per
// primitive quartet, the block written back lane-strided.
template <int LA, int LB, int LC, int LD>
__global__ void __launch_bounds__(32 * kColWarps) col_prim_kernel(const PrimQuartetParams prm) {
  using S = ColSmem<double, LA, LB, LC, LD>;
  extern __shared__ __align__(16) unsigned char col_smraw[];
  S* sm = reinterpret_cast<S*>(col_smraw) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  const long long q = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (q >= prm.n) return;
  for (int i = lane; i < int(sizeof(sm->Fk) / sizeof(double)); i += 32) (&sm->Fk[0][0][0][0])[i] = 0.0;
  for (int i = lane; i < int(sizeof(sm->Eb) / sizeof(double)); i += 32) (&sm->Eb[0][0][0][0])[i] = 0.0;
  for (int i = lane; i < S::NAB * S::NCD; i += 32) sm->blk[i] = 0.0;
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
  __syncwarp();
  col_set_bra<double, LA, LB, LC, LD>(sm, bra, A, B, lane);
  col_add_prim<double, LA, LB, LC, LD>(sm, bra, ket, C, D, prm.boys, lane);
  double* o = prm.out + q * (S::NAB * S::NCD);
  for (int x = lane; x < S::NAB * S::NCD; x += 32) o[x] = sm->blk[x];
}

template <int LA, int LB, int LC, int LD>
static cudaError_t launch_col_prim_class(const PrimQuartetParams& p, cudaStream_t s) {
  if (p.n == 0) return cudaSuccess;
  const size_t sm = kColWarps * sizeof(ColSmem<double, LA, LB, LC, LD>);
  static bool configured = false;
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(col_prim_kernel<LA, LB, LC, LD>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    configured = true;
  }
  const unsigned grid = (unsigned)((p.n + kColWarps - 1) / kColWarps);
  col_prim_kernel<LA, LB, LC, LD><<<grid, 32 * kColWarps, sm, s>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_col_prim(int qc, const PrimQuartetParams& p, cudaStream_t s) {
  switch (qc) {
    case 19:
      return launch_col_prim_class<2, 2, 2, 1>(p, s);
    case 20:
      return launch_col_prim_class<2, 2, 2, 2>(p, s);
    default:
      return cudaErrorNotSupported;
  }
}

// Classes with a column-engine kernel.
#define JQC_FOR_COL_CLASSES(X) \
  X(12, 2, 1, 1, 1)            \
  X(13, 2, 1, 2, 0)            \
  X(14, 2, 1, 2, 1)            \
  X(16, 2, 2, 1, 0)            \
  X(17, 2, 2, 1, 1)            \
  X(18, 2, 2, 2, 0)            \
  X(19, 2, 2, 2, 1)            \
  X(20, 2, 2, 2, 2)

bool has_col_class(int qc) {
  switch (qc) {
#define X(Q, A, B, C, D) case Q:
    JQC_FOR_COL_CLASSES(X)
#undef X
    return true;
    default:
      return false;
  }
}

cudaError_t launch_col_jk(int qc, bool fp32, const JKParams& p, cudaStream_t s) {
  switch (qc) {
#define X(Q, A, B, C, D) \
  case Q:                \
    return fp32 ? launch_col_jk_class<float, A, B, C, D>(p, s) : launch_col_jk_class<double, A, B, C, D>(p, s);
    JQC_FOR_COL_CLASSES(X)
#undef X
    default:
      return cudaErrorNotSupported;
  }
}

}  // namespace jqc
