// McMurchie-Davidson machinery for contracted shell quartets on the device.
//
// The algorithm is the reference's (jax_qc/integrals/obara_saika.py:227-332,
// mcmurchie_davidson.py:60-172):
//   (ab|cd) = 2 pi^{5/2} / (p q sqrt(p+q)) K_AB K_CD
//             sum_{tuv} E^{ab}_{tuv} sum_{t'u'v'} (-1)^{t'+u'+v'} E^{cd}_{t'u'v'}
//             R_{t+t', u+u', v+v'}(rho, P-Q)
// restructured for registers: everything is unrolled at compile time for one
// angular class (LA LB | LC LD); the R_tuv^n recursion runs in place over n
// (one array of C(L+3,3) values); the Hermite contraction is done in two
// stages, first over the ket Hermite index into X_tuv for one ket Cartesian
// pair, then over the bra Hermite index into the output block.
#pragma once

#include "boys.cuh"
#include "common.cuh"

namespace jqc {

// One primitive pair of a shell pair (a, b): p = alpha + beta,
// P = (alpha A + beta B) / p, K = exp(-alpha beta |AB|^2 / p) c_a c_b,
// h = 1/(2p) (kept so no kernel divides by p).  32-byte aligned: the records
// live in cudaMalloc'd arrays and are read with 32-byte vector loads.
struct __align__(32) PrimPair {
  double p, h, Px, Py, Pz, K, alpha, beta;
};
struct __align__(32) PrimPairF {
  float p, h, Px, Py, Pz, K, alpha, beta;
};
static_assert(sizeof(PrimPair) == 64 && sizeof(PrimPairF) == 32, "primitive-pair records");

// 32-byte vector loads of a primitive-pair record through the read-only path
// (global memory only; records built in registers/local memory are read
// with plain loads, see quartet_accumulate's GLOBAL_PP).
__device__ __forceinline__ PrimPair ld_pp(const PrimPair* q) {
  const double* v = reinterpret_cast<const double*>(q);
  PrimPair r;
  ldg32B(v, r.p, r.h, r.Px, r.Py);
  ldg32B(v + 4, r.Pz, r.K, r.alpha, r.beta);
  return r;
}
__device__ __forceinline__ PrimPairF ld_pp(const PrimPairF* q) {
  float v[8];
  ldg32B(reinterpret_cast<const float*>(q), v);
  return PrimPairF{v[0], v[1], v[2], v[3], v[4], v[5], v[6], v[7]};
}
template <typename T>
struct PPType;
template <>
struct PPType<double> {
  using type = PrimPair;
};
template <>
struct PPType<float> {
  using type = PrimPairF;
};

// Shell pair (a, b) with la >= lb.  pp/npp index its primitive pairs.
struct __align__(16) ShellPair {
  int a, b, pp, npp;
  double Q;    // Schwarz bound sqrt(max (ab|ab))
  int diag;    // a == b
  int cls;     // angular pair class
};

// Work item: one bra pair against a run of at most 32 consecutive ket pairs.
struct __align__(16) Task {
  int bra, ket0, nket, flags;
};

constexpr double kTwoPi25 = 34.986836655249725693;  // 2 pi^{5/2}

// ---------------------------------------------------------------- E coeffs

// E^{ij}_t along one axis for i <= LA, j <= LB (E^{00}_0 = 1), by
//   E^{i+1,j}_t = E^{ij}_{t-1}/(2p) + X_PA E^{ij}_t + (t+1) E^{ij}_{t+1}
//   E^{i,j+1}_t = E^{ij}_{t-1}/(2p) + X_PB E^{ij}_t + (t+1) E^{ij}_{t+1}
// (mcmurchie_davidson.py:60-108).  With SIGN the coefficients carry
// (-1)^t (the ket side of the contraction).
template <typename T, int LA, int LB>
using EArr = T (*)[LB + 1][LA + LB + 1];

template <typename T, int LA, int LB, bool SIGN>
__device__ __forceinline__ void ecoef_compute(EArr<T, LA, LB> e, T pa, T pb, T inv2p) {
  e[0][0][0] = T(1);
  static_for<LA>([&](auto ii) {
    constexpr int i = decltype(ii)::value;
    static_for<i + 2>([&](auto tt) {
      constexpr int t = decltype(tt)::value;
      T v = T(0);
      if constexpr (t <= i) v = pa * e[i][0][t];
      if constexpr (t >= 1) v += inv2p * e[i][0][t - 1];
      if constexpr (t + 1 <= i) v += T(t + 1) * e[i][0][t + 1];
      e[i + 1][0][t] = v;
    });
  });
  static_for<LB>([&](auto jj) {
    constexpr int j = decltype(jj)::value;
    static_for<LA + 1>([&](auto ii) {
      constexpr int i = decltype(ii)::value;
      static_for<i + j + 2>([&](auto tt) {
        constexpr int t = decltype(tt)::value;
        T v = T(0);
        if constexpr (t <= i + j) v = pb * e[i][j][t];
        if constexpr (t >= 1) v += inv2p * e[i][j][t - 1];
        if constexpr (t + 1 <= i + j) v += T(t + 1) * e[i][j][t + 1];
        e[i][j + 1][t] = v;
      });
    });
  });
  if constexpr (SIGN) {
    static_for<LA + 1>([&](auto ii) {
      static_for<LB + 1>([&](auto jj) {
        constexpr int i = decltype(ii)::value, j = decltype(jj)::value;
        static_for<(i + j + 1) / 2>([&](auto kk) {
          constexpr int t = 2 * decltype(kk)::value + 1;
          e[i][j][t] = -e[i][j][t];
        });
      });
    });
  }
}

// ---------------------------------------------------------------- R_tuv

// In-place R recursion.  On entry Rn[n] = pref * (-2 rho)^n F_n(T), n <= L.
// On exit R[herm_index(t,u,v)] = pref * R^0_{tuv} for t+u+v <= L.
// Level n is built from level n+1 by t/u/v raising (Helgaker 9.9.18-20);
// within a level, higher total orders are written first so every read sees
// level n+1 values.
template <typename T, int L>
__device__ __forceinline__ void hermite_R(T (&R)[nherm(L)], const T (&Rn)[L + 1], T X, T Y, T Z) {
  R[0] = Rn[L];
  static_for<L>([&](auto nn) {
    constexpr int n = L - 1 - decltype(nn)::value;
    static_for<L - n>([&](auto ss) {
      constexpr int s = L - n - decltype(ss)::value;
      static_for<ncart(s)>([&](auto kk) {
        constexpr int k = decltype(kk)::value;
        constexpr int t = cart_lx(s, k), u = cart_ly(s, k), v = s - t - u;
        T val;
        if constexpr (t > 0) {
          val = X * R[herm_index(t - 1, u, v)];
          if constexpr (t > 1) val += T(t - 1) * R[herm_index(t - 2, u, v)];
        } else if constexpr (u > 0) {
          val = Y * R[herm_index(t, u - 1, v)];
          if constexpr (u > 1) val += T(u - 1) * R[herm_index(t, u - 2, v)];
        } else {
          val = Z * R[herm_index(t, u, v - 1)];
          if constexpr (v > 1) val += T(v - 1) * R[herm_index(t, u, v - 2)];
        }
        R[herm_index(t, u, v)] = val;
      });
    });
    R[0] = Rn[n];
  });
}

// ------------------------------------------------------------ quartet core

template <int LA, int LB, int LC, int LD, int NS, int PART>
struct QCfg {
  static constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
  static constexpr int NAB = NA * NB, NCD = NC * ND;
  static constexpr int CDP = (NCD + NS - 1) / NS;  // ket Cartesian pairs per part
  static constexpr int CD0 = PART * CDP;
  static constexpr int NCDP = (CD0 >= NCD) ? 0 : ((CD0 + CDP <= NCD) ? CDP : NCD - CD0);
  static constexpr int L = LA + LB + LC + LD;
  static constexpr int LAB = LA + LB;
};

template <typename T>
struct Vec3 {
  T x, y, z;
};

__device__ __forceinline__ double fast_rsqrt(double x) { return rsqrt(x); }
__device__ __forceinline__ float fast_rsqrt(float x) { return rsqrtf(x); }

// Primitive-quartet scalars: fills Rn[n] = pref (-2 rho)^n F_n and R.
template <typename T, int L, typename PPT>
__device__ __forceinline__ void prim_quartet_R(const PPT& bp, const PPT& kp, const T* __restrict__ boys_tab,
                                               T (&R)[nherm(L)]) {
  // 1/(p+q) = r^2 with r = 1/sqrt(p+q); 1/(pq) = 4 h_p h_q: no divisions.
  const T p = bp.p, q = kp.p;
  const T r = fast_rsqrt(p + q);
  const T rho = p * q * (r * r);
  const T PQx = bp.Px - kp.Px, PQy = bp.Py - kp.Py, PQz = bp.Pz - kp.Pz;
  const T tb = rho * (PQx * PQx + PQy * PQy + PQz * PQz);
  T F[L + 1];
  boys_eval<T, L>(tb, boys_tab, F);
  T pref = T(4.0 * kTwoPi25) * T(bp.K) * T(kp.K) * (T(bp.h) * T(kp.h)) * r;
  T Rn[L + 1];
  const T m2rho = T(-2) * rho;
  static_for<L + 1>([&](auto nn) {
    constexpr int n = decltype(nn)::value;
    Rn[n] = pref * F[n];
    pref *= m2rho;
  });
  hermite_R<T, L>(R, Rn, PQx, PQy, PQz);
}

// Classes whose bra angular sum is at most this loop over ket primitives
// outermost (see quartet_accumulate) and read their bra per lane, so the
// register J/K kernel can pack the kets of several bra pairs into one warp.
constexpr int kKetOuterMaxLab = 2;

// Accumulates the contracted block (ab|cd) for the ket Cartesian pairs of
// part PART into out[ab][cdi] (cd = CD0 + cdi).  Loops over all primitive
// pairs of the bra (outer) and ket (inner) shell pairs.  The bra E
// coefficients live in `ebra` (3 axes); with SHARED_BRA the bra pair is the
// same for the whole warp, `ebra` is warp-private shared memory and lanes
// 0..2 fill one axis each (every lane of the warp must call this function).
// GLOBAL_PP: bra/ket point into global memory (vector read-only loads);
// false for primitive pairs built on the fly by the caller.
template <typename T, int LA, int LB, int LC, int LD, int NS, int PART, bool SHARED_BRA, bool GLOBAL_PP = true>
__device__ __forceinline__ void quartet_accumulate(
    const typename PPType<T>::type* __restrict__ bra, int nbra, Vec3<T> A, Vec3<T> B,
    const typename PPType<T>::type* __restrict__ ket, int nket, Vec3<T> C, Vec3<T> D,
    const T* __restrict__ boys_tab, T (*ebra)[LA + 1][LB + 1][LA + LB + 1],
    T (&out)[QCfg<LA, LB, LC, LD, NS, PART>::NAB][QCfg<LA, LB, LC, LD, NS, PART>::CDP]) {
  using Cfg = QCfg<LA, LB, LC, LD, NS, PART>;
  constexpr int L = Cfg::L;
  constexpr int LAB = Cfg::LAB;
  static_for<Cfg::NAB>([&](auto ab) {
    static_for<Cfg::CDP>([&](auto c) { out[decltype(ab)::value][decltype(c)::value] = T(0); });
  });
  if constexpr (Cfg::NCDP > 0) {
    using PPT = typename PPType<T>::type;
    // One primitive quartet: R, stage 1 (ket E against R) and stage 2 (bra E).
    auto prim = [&](const PPT& bp, const EArr<T, LA, LB> Ex, const EArr<T, LA, LB> Ey, const EArr<T, LA, LB> Ez,
                    const PPT& kp, const EArr<T, LC, LD> Fx, const EArr<T, LC, LD> Fy, const EArr<T, LC, LD> Fz) {
      T R[nherm(L)];
      prim_quartet_R<T, L>(bp, kp, boys_tab, R);
      static_for<Cfg::NCDP>([&](auto cdi_) {
        constexpr int cdi = decltype(cdi_)::value;
        constexpr int cd = Cfg::CD0 + cdi, c = cd / Cfg::ND, d = cd % Cfg::ND;
        constexpr int cx = cart_lx(LC, c), cy = cart_ly(LC, c), cz = cart_lz(LC, c);
        constexpr int dx = cart_lx(LD, d), dy = cart_ly(LD, d), dz = cart_lz(LD, d);
        // stage 1: X_tuv = sum_{t'u'v'} F^x F^y F^z R_{t+t',u+u',v+v'}
        T X[nherm(LAB)];
        static_for<nherm(LAB)>([&](auto h) { X[decltype(h)::value] = T(0); });
        static_for<cx + dx + 1>([&](auto tp_) {
          constexpr int tp = decltype(tp_)::value;
          static_for<cy + dy + 1>([&](auto up_) {
            constexpr int up = decltype(up_)::value;
            const T fxy = Fx[cx][dx][tp] * Fy[cy][dy][up];
            static_for<cz + dz + 1>([&](auto vp_) {
              constexpr int vp = decltype(vp_)::value;
              const T f = fxy * Fz[cz][dz][vp];
              static_for<nherm(LAB)>([&](auto h_) {
                constexpr int h = decltype(h_)::value;
                constexpr int s = (h >= 20) ? 4 : (h >= 10) ? 3 : (h >= 4) ? 2 : (h >= 1) ? 1 : 0;
                constexpr int k = h - s * (s + 1) * (s + 2) / 6;
                constexpr int t = cart_lx(s, k), u = cart_ly(s, k), v = s - t - u;
                X[h] += f * R[herm_index(t + tp, u + up, v + vp)];
              });
            });
          });
        });
        // stage 2: out[ab][cd] += sum_tuv E^x E^y E^z X_tuv
        static_for<Cfg::NA>([&](auto a_) {
          constexpr int a = decltype(a_)::value;
          constexpr int ax = cart_lx(LA, a), ay = cart_ly(LA, a), az = cart_lz(LA, a);
          static_for<Cfg::NB>([&](auto b_) {
            constexpr int b = decltype(b_)::value;
            constexpr int bx = cart_lx(LB, b), by = cart_ly(LB, b), bz = cart_lz(LB, b);
            T acc = T(0);
            static_for<ax + bx + 1>([&](auto t_) {
              constexpr int t = decltype(t_)::value;
              static_for<ay + by + 1>([&](auto u_) {
                constexpr int u = decltype(u_)::value;
                const T exy = Ex[ax][bx][t] * Ey[ay][by][u];
                static_for<az + bz + 1>([&](auto v_) {
                  constexpr int v = decltype(v_)::value;
                  acc += exy * Ez[az][bz][v] * X[herm_index(t, u, v)];
                });
              });
            });
            out[a * Cfg::NB + b][cdi] += acc;
          });
        });
      });
    };
    auto ket_e = [&](const PPT& kp, T (*fbuf)[LC + 1][LD + 1][LC + LD + 1]) {
      ecoef_compute<T, LC, LD, true>(fbuf[0], kp.Px - C.x, kp.Px - D.x, kp.h);
      ecoef_compute<T, LC, LD, true>(fbuf[1], kp.Py - C.y, kp.Py - D.y, kp.h);
      ecoef_compute<T, LC, LD, true>(fbuf[2], kp.Pz - C.z, kp.Pz - D.z, kp.h);
    };
    if constexpr (GLOBAL_PP && LA + LB <= kKetOuterMaxLab) {
      // Ket primitives outer: each lane reads its ket primitive pair and its
      // E coefficients once; the bra primitive pairs (the same address in
      // every lane: one broadcast read) and their few E coefficients are
      // redone per ket primitive in registers.  Cuts the per-lane global
      // reads of the low-L classes, which are bound by L1 throughput.
      for (int iq = 0; iq < nket; ++iq) {
        const PPT kp = ld_pp(ket + iq);
        T fbuf[3][LC + 1][LD + 1][LC + LD + 1];
        ket_e(kp, fbuf);
        for (int ip = 0; ip < nbra; ++ip) {
          const PPT bp = ld_pp(bra + ip);
          T eb[3][LA + 1][LB + 1][LA + LB + 1];
          ecoef_compute<T, LA, LB, false>(eb[0], bp.Px - A.x, bp.Px - B.x, bp.h);
          ecoef_compute<T, LA, LB, false>(eb[1], bp.Py - A.y, bp.Py - B.y, bp.h);
          ecoef_compute<T, LA, LB, false>(eb[2], bp.Pz - A.z, bp.Pz - B.z, bp.h);
          prim(bp, eb[0], eb[1], eb[2], kp, fbuf[0], fbuf[1], fbuf[2]);
        }
      }
    } else {
      const int lane = threadIdx.x & 31;
      for (int ip = 0; ip < nbra; ++ip) {
        PPT bp;
        if constexpr (GLOBAL_PP) bp = ld_pp(bra + ip);
        else bp = bra[ip];
        const T inv2p = bp.h;
        if constexpr (SHARED_BRA) {
          __syncwarp();
          if (lane == 0) ecoef_compute<T, LA, LB, false>(ebra[0], bp.Px - A.x, bp.Px - B.x, inv2p);
          if (lane == 1) ecoef_compute<T, LA, LB, false>(ebra[1], bp.Py - A.y, bp.Py - B.y, inv2p);
          if (lane == 2) ecoef_compute<T, LA, LB, false>(ebra[2], bp.Pz - A.z, bp.Pz - B.z, inv2p);
          __syncwarp();
        } else {
          ecoef_compute<T, LA, LB, false>(ebra[0], bp.Px - A.x, bp.Px - B.x, inv2p);
          ecoef_compute<T, LA, LB, false>(ebra[1], bp.Py - A.y, bp.Py - B.y, inv2p);
          ecoef_compute<T, LA, LB, false>(ebra[2], bp.Pz - A.z, bp.Pz - B.z, inv2p);
        }
        for (int iq = 0; iq < nket; ++iq) {
          PPT kp;
          if constexpr (GLOBAL_PP) kp = ld_pp(ket + iq);
          else kp = ket[iq];
          T fbuf[3][LC + 1][LD + 1][LC + LD + 1];
          ket_e(kp, fbuf);
          prim(bp, ebra[0], ebra[1], ebra[2], kp, fbuf[0], fbuf[1], fbuf[2]);
        }
      }
    }
  }
}

// Dispatch a runtime part index (uniform over the block: blockIdx.y) to the
// compile-time PART of a functor template.
#define JQC_PART_CASE(P)                                    \
  case P:                                                   \
    if constexpr (P < NS) f.template run<P>();             \
    break;
template <int NS, typename F>
__device__ __forceinline__ void dispatch_part(int part, F& f) {
  switch (part) {
    JQC_PART_CASE(0) JQC_PART_CASE(1) JQC_PART_CASE(2) JQC_PART_CASE(3)
    JQC_PART_CASE(4) JQC_PART_CASE(5) JQC_PART_CASE(6) JQC_PART_CASE(7)
    JQC_PART_CASE(8) JQC_PART_CASE(9) JQC_PART_CASE(10) JQC_PART_CASE(11)
    JQC_PART_CASE(12) JQC_PART_CASE(13) JQC_PART_CASE(14) JQC_PART_CASE(15)
    default: break;
  }
}
#undef JQC_PART_CASE

// Number of parts the ket Cartesian pairs of a class are split into, so that
// one thread holds at most ~40 accumulators.
__host__ __device__ constexpr int class_split(int la, int lb, int lc, int ld) {
  int nab = ncart(la) * ncart(lb), ncd = ncart(lc) * ncart(ld);
  int ns = 1;
  while (ns < 16 && nab * ((ncd + ns - 1) / ns) > 40 && ns < ncd) ns *= 2;
  return ns;
}

}  // namespace jqc
