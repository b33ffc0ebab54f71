// Warp-cooperative engine for the high angular-momentum classes (L >= 5:
// quartets with d shells on both sides).  One warp evaluates one contracted
// shell quartet at a time with the class given at run time:
//   * lanes 0..L evaluate F_m(T) directly from the Boys table (Taylor at
//     order m), so no recursion over m is serial;
//   * the R_tuv^n recursion runs in shared memory, one total order at a
//     time, lanes parallel over the entries of that order;
//   * lanes 0..5 build the bra / ket E coefficients (one axis each);
//   * stage 1 (ket Hermite -> X[cd][tuv]) and stage 2 (bra Hermite ->
//     block[ab][cd]) are spread over the lanes; block elements stay in
//     registers (lane owns elements lane, lane+32, ...).
// The same body serves J/K digestion, the dense tensor, Schwarz bounds and
// primitive blocks (MODE).
#pragma once

#include "kernels.cuh"

namespace jqc {

// One step of the in-place Hermite recursion for each Hermite index h of
// total order s >= 1 (t, u, v): R_h = PQ_axis R_src1 + coef R_src2 along the
// first axis with a nonzero index (R_{t,u,v} = X R_{t-1,u,v} + (t-1)
// R_{t-2,u,v}, ...), packed as src1 | src2 << 9 | coef << 18 | axis << 22
// (src2 = coef = 0 where the second term is absent).  Built at compile time;
// the warp recursions below read one code per lane and order instead of
// decoding (t, u, v) with integer loops.
constexpr int kRCodeMaxL = 10;
struct RCodeTable {
  int v[nherm(kRCodeMaxL)];
  constexpr RCodeTable() : v() {
    for (int s = 1; s <= kRCodeMaxL; ++s)
      for (int k = 0; k < ncart(s); ++k) {
        const int t = cart_lx(s, k), u = cart_ly(s, k), w = s - t - u;
        int ax = 2, s1 = 0, s2 = 0, cf = 0;
        if (t > 0) {
          ax = 0;
          s1 = herm_index(t - 1, u, w);
          if (t > 1) s2 = herm_index(t - 2, u, w), cf = t - 1;
        } else if (u > 0) {
          ax = 1;
          s1 = herm_index(t, u - 1, w);
          if (u > 1) s2 = herm_index(t, u - 2, w), cf = u - 1;
        } else {
          s1 = herm_index(t, u, w - 1);
          if (w > 1) s2 = herm_index(t, u, w - 2), cf = w - 1;
        }
        v[nherm(s - 1) + k] = s1 | (s2 << 9) | (cf << 18) | (ax << 22);
      }
  }
};
__device__ constexpr RCodeTable kRCode{};

// R^0_tuv for all t+u+v <= L into R (warp-shared, Hermite layout) from
// Rn[n] = R^n_000, in place: level n = L-1 .. 0, order s = L-n .. 1 (highest
// first, so the lower orders still hold level n+1), lanes over the
// components of one order.  Fully unrolled; each lane keeps its recursion
// codes in registers.
template <typename T, int L>
__device__ __forceinline__ void warp_hermite_R(T* R, const T* Rn, T X, T Y, T Z, int lane) {
  static_assert(L <= kRCodeMaxL, "recursion table too small");
  int code[L + 1][2];
  static_for<L>([&](auto i_) {
    constexpr int s = decltype(i_)::value + 1;
    code[s][0] = lane < ncart(s) ? __ldg(kRCode.v + nherm(s - 1) + lane) : 0;
    code[s][1] = lane + 32 < ncart(s) ? __ldg(kRCode.v + nherm(s - 1) + lane + 32) : 0;
  });
  if (lane == 0) R[0] = Rn[L];
  __syncwarp();
  static_for<L>([&](auto i_) {
    constexpr int n = L - 1 - decltype(i_)::value;
    static_for<L - n>([&](auto j_) {
      constexpr int s = L - n - decltype(j_)::value;
      static_for<(ncart(s) + 31) / 32>([&](auto r_) {
        constexpr int r = decltype(r_)::value;
        const int k = 32 * r + lane;
        if (k < ncart(s)) {
          const int c = code[s][r];
          const int ax = c >> 22;
          const T pq = ax == 0 ? X : (ax == 1 ? Y : Z);
          R[nherm(s - 1) + k] = pq * R[c & 511] + T((c >> 18) & 15) * R[(c >> 9) & 511];
        }
      });
      __syncwarp();
    });
    if (lane == 0) R[0] = Rn[n];
    __syncwarp();
  });
}

constexpr int kWarpMaxL = 8;
constexpr int kWarpMaxHerm = nherm(kWarpMaxL);          // 165
constexpr int kWarpMaxHab = nherm(4);                    // 35 bra Hermite functions
constexpr int kWarpMaxBlock = 36 * 36;                   // (dd|dd)
constexpr int kWarpSlots = (kWarpMaxBlock + 31) / 32;    // 41 elements per lane

template <typename T>
struct WarpSmem {
  T R[kWarpMaxHerm];
  T Rn[kWarpMaxL + 2];
  T E[2][3][3][3][5];       // [bra/ket][axis][i][j][t]; ket carries (-1)^t
  T XB[kWarpMaxBlock];      // stage-1 X[cd][h]; later the finished block
};

enum WarpMode { kWarpJK = 0, kWarpTensor = 1, kWarpSchwarz = 2, kWarpPrim = 3 };

struct WarpParams {
  int la, lb, lc, ld;
  JKParams jk;            // JK mode (tasks, pairs, pp, centres, ao, boys, D/J/K...)
  double* eri;            // tensor mode
  long long n_tensor;
  const int* pair_ids;    // Schwarz mode
  unsigned long long* qmax;
  const double* exps;     // prim mode
  const double* pcentres;
  double* pout;
  long long n_prim;
};

__device__ __forceinline__ int wcart_lx(int l, int k) {
  int lx = l;
  while (k > l - lx) {
    k -= (l - lx + 1);
    --lx;
  }
  return lx;
}
__device__ __forceinline__ void wcart(int l, int k, int& x, int& y, int& z) {
  int lx = l;
  while (k > l - lx) {
    k -= (l - lx + 1);
    --lx;
  }
  x = lx;
  y = (l - lx) - k;
  z = l - x - y;
}
__device__ __forceinline__ void wherm(int h, int& t, int& u, int& v) {
  int s = 0;
  while ((s + 1) * (s + 2) * (s + 3) / 6 <= h) ++s;
  wcart(s, h - s * (s + 1) * (s + 2) / 6, t, u, v);
}

// E coefficients along one axis with runtime la, lb into e[i][j][t].
template <typename T>
__device__ __forceinline__ void wecoef(T (*e)[3][5], int la, int lb, T pa, T pb, T inv2p, bool sign) {
  for (int i = 0; i <= la; ++i)
    for (int j = 0; j <= lb; ++j)
      for (int t = 0; t < 5; ++t) e[i][j][t] = T(0);
  e[0][0][0] = T(1);
  for (int i = 0; i < la; ++i)
    for (int t = 0; t <= i + 1; ++t) {
      T v = T(0);
      if (t <= i) v = pa * e[i][0][t];
      if (t >= 1) v += inv2p * e[i][0][t - 1];
      if (t + 1 <= i) v += T(t + 1) * e[i][0][t + 1];
      e[i + 1][0][t] = v;
    }
  for (int j = 0; j < lb; ++j)
    for (int i = 0; i <= la; ++i)
      for (int t = 0; t <= i + j + 1; ++t) {
        T v = T(0);
        if (t <= i + j) v = pb * e[i][j][t];
        if (t >= 1) v += inv2p * e[i][j][t - 1];
        if (t + 1 <= i + j) v += T(t + 1) * e[i][j][t + 1];
        e[i][j + 1][t] = v;
      }
  if (sign)
    for (int i = 0; i <= la; ++i)
      for (int j = 0; j <= lb; ++j)
        for (int t = 1; t < 5; t += 2) e[i][j][t] = -e[i][j][t];
}

// F_m(T) for one m straight from the table (T < TMax) or by upward
// recursion from the asymptotic F_0 (T >= TMax).
template <typename T>
__device__ __forceinline__ T boys_single(T t, int m, const T* __restrict__ tab) {
  constexpr int KT = BoysConst<T>::kTaylor;
  if (t < T(kBoysTMax)) {
    const int i = boys_round(t * T(kBoysGridInv));
    const T d = T(i) * T(1.0 / kBoysGridInv) - t;
    const T* row = tab + i * kBoysCols + m;
    T acc = __ldg(row + KT - 1);
#pragma unroll
    for (int k = KT - 2; k >= 0; --k) acc = __ldg(row + k) + acc * (d * T(1.0 / (k + 1)));
    return acc;
  }
  const T inv_t = T(1) / t;
  T f = T(0.88622692545275801364908374167057) * boys_sqrt(inv_t);
  const T e = boys_exp(-t);
  for (int k = 0; k < m; ++k) f = (T(2 * k + 1) * f - e) * T(0.5) * inv_t;
  return f;
}

template <typename T>
struct WarpQuartet {
  WarpSmem<T>* sm;
  int lane;
  int la, lb, lc, ld, L, nab, ncd, nhab, ntot;
  T acc[kWarpSlots];

  __device__ __forceinline__ void init(int la_, int lb_, int lc_, int ld_) {
    la = la_;
    lb = lb_;
    lc = lc_;
    ld = ld_;
    L = la + lb + lc + ld;
    nab = ncart(la) * ncart(lb);
    ncd = ncart(lc) * ncart(ld);
    nhab = nherm(la + lb);
    ntot = nab * ncd;
#pragma unroll
    for (int k = 0; k < kWarpSlots; ++k) acc[k] = T(0);
  }

  // Bra E for one bra primitive pair (all lanes call).
  __device__ __forceinline__ void set_bra(T Px, T Py, T Pz, T hp, Vec3<T> A, Vec3<T> B) {
    __syncwarp();
    const T inv2p = hp;
    if (lane == 0) wecoef<T>(sm->E[0][0], la, lb, Px - A.x, Px - B.x, inv2p, false);
    if (lane == 1) wecoef<T>(sm->E[0][1], la, lb, Py - A.y, Py - B.y, inv2p, false);
    if (lane == 2) wecoef<T>(sm->E[0][2], la, lb, Pz - A.z, Pz - B.z, inv2p, false);
  }

  // One primitive quartet (all lanes call with the same arguments).
  __device__ __forceinline__ void add_prim(T p, T hp, T Px, T Py, T Pz, T Kab, T q, T hq, T Qx, T Qy, T Qz, T Kcd,
                                           Vec3<T> C, Vec3<T> D, const T* __restrict__ tab) {
    const T inv2q = hq;
    if (lane == 3) wecoef<T>(sm->E[1][0], lc, ld, Qx - C.x, Qx - D.x, inv2q, true);
    if (lane == 4) wecoef<T>(sm->E[1][1], lc, ld, Qy - C.y, Qy - D.y, inv2q, true);
    if (lane == 5) wecoef<T>(sm->E[1][2], lc, ld, Qz - C.z, Qz - D.z, inv2q, true);
    const T r = fast_rsqrt(p + q);
    const T rho = p * q * (r * r);
    const T X = Px - Qx, Y = Py - Qy, Z = Pz - Qz;
    const T tb = rho * (X * X + Y * Y + Z * Z);
    if (lane <= L) {
      T pref = T(4.0 * kTwoPi25) * Kab * Kcd * (hp * hq) * r;
      const T m2rho = T(-2) * rho;
      for (int k = 0; k < lane; ++k) pref *= m2rho;
      sm->Rn[lane] = pref * boys_single<T>(tb, lane, tab);
    }
    __syncwarp();
    // in-place R recursion over n (see hermite_R in mmd.cuh)
    if (lane == 0) sm->R[0] = sm->Rn[L];
    __syncwarp();
    for (int n = L - 1; n >= 0; --n) {
      for (int s = L - n; s >= 1; --s) {
        const int base = s * (s + 1) * (s + 2) / 6;
        for (int k = lane; k < ncart(s); k += 32) {
          int t, u, v;
          wcart(s, k, t, u, v);
          T val;
          if (t > 0) {
            val = X * sm->R[herm_index(t - 1, u, v)];
            if (t > 1) val += T(t - 1) * sm->R[herm_index(t - 2, u, v)];
          } else if (u > 0) {
            val = Y * sm->R[herm_index(t, u - 1, v)];
            if (u > 1) val += T(u - 1) * sm->R[herm_index(t, u - 2, v)];
          } else {
            val = Z * sm->R[herm_index(t, u, v - 1)];
            if (v > 1) val += T(v - 1) * sm->R[herm_index(t, u, v - 2)];
          }
          sm->R[base + k] = val;
        }
        __syncwarp();
      }
      if (lane == 0) sm->R[0] = sm->Rn[n];
      __syncwarp();
    }
    // stage 1: X[cd][h]
    const int nd = ncart(ld);
    for (int idx = lane; idx < ncd * nhab; idx += 32) {
      const int cd = idx / nhab, h = idx % nhab;
      int t, u, v, cx, cy, cz, dx, dy, dz;
      wherm(h, t, u, v);
      wcart(lc, cd / nd, cx, cy, cz);
      wcart(ld, cd % nd, dx, dy, dz);
      T x = T(0);
      for (int tp = 0; tp <= cx + dx; ++tp)
        for (int up = 0; up <= cy + dy; ++up) {
          const T fxy = sm->E[1][0][cx][dx][tp] * sm->E[1][1][cy][dy][up];
          for (int vp = 0; vp <= cz + dz; ++vp)
            x += fxy * sm->E[1][2][cz][dz][vp] * sm->R[herm_index(t + tp, u + up, v + vp)];
        }
      sm->XB[idx] = x;
    }
    __syncwarp();
    // stage 2: block elements owned by this lane
    const int nb = ncart(lb);
#pragma unroll
    for (int k = 0; k < kWarpSlots; ++k) {
      const int e = lane + 32 * k;
      if (e < ntot) {
        const int ab = e / ncd, cd = e % ncd;
        int ax, ay, az, bx, by, bz;
        wcart(la, ab / nb, ax, ay, az);
        wcart(lb, ab % nb, bx, by, bz);
        T s = T(0);
        for (int t = 0; t <= ax + bx; ++t)
          for (int u = 0; u <= ay + by; ++u) {
            const T exy = sm->E[0][0][ax][bx][t] * sm->E[0][1][ay][by][u];
            for (int v = 0; v <= az + bz; ++v)
              s += exy * sm->E[0][2][az][bz][v] * sm->XB[cd * nhab + herm_index(t, u, v)];
          }
        acc[k] += s;
      }
    }
    __syncwarp();
  }

  // Block to shared memory (XB), all lanes call.
  __device__ __forceinline__ void publish() {
    __syncwarp();
#pragma unroll
    for (int k = 0; k < kWarpSlots; ++k) {
      const int e = lane + 32 * k;
      if (e < ntot) sm->XB[e] = acc[k];
    }
    __syncwarp();
  }
};

// J/K digestion of one finished contracted block blk[ab * ncd + cd] (shared
// memory, all lanes call) with scale s: J[a][b] and J[c][d] (Coulomb of both
// pairs) and the four exchange blocks K[a][d], K[a][c], K[b][d], K[b][c],
// lanes spread over output elements, one atomic per element.
template <typename T>
__device__ __forceinline__ void warp_digest_jk(const JKParams& prm, const T* blk, int na, int nb, int nc, int nd,
                                               int a0, int b0, int c0, int d0, double s, int lane) {
  const int n = prm.n;
  const int ncd = nc * nd;
  for (int dd = 0; dd < prm.n_dens; ++dd) {
    const double* Dm = prm.D + (size_t)dd * n * n;
    double* Jm = prm.J + (size_t)dd * n * n;
    double* Km = prm.K + (size_t)dd * n * n;
    for (int ab = lane; ab < na * nb; ab += 32) {
      double acc = 0.0;
      for (int cd = 0; cd < ncd; ++cd)
        acc += double(blk[ab * ncd + cd]) * __ldg(Dm + (size_t)(c0 + cd / nd) * n + d0 + cd % nd);
      atomicAdd(Jm + (size_t)(a0 + ab / nb) * n + b0 + ab % nb, 2.0 * s * acc);
    }
    for (int cd = lane; cd < ncd; cd += 32) {
      double acc = 0.0;
      for (int ab = 0; ab < na * nb; ++ab)
        acc += double(blk[ab * ncd + cd]) * __ldg(Dm + (size_t)(a0 + ab / nb) * n + b0 + ab % nb);
      atomicAdd(Jm + (size_t)(c0 + cd / nd) * n + d0 + cd % nd, 2.0 * s * acc);
    }
    // K[a][d] += v D[c][b]; K[a][c] += v D[d][b]
    for (int idx = lane; idx < na * (nd + nc); idx += 32) {
      const int a = idx / (nd + nc), r = idx % (nd + nc);
      double acc = 0.0;
      if (r < nd) {
        for (int b = 0; b < nb; ++b)
          for (int c = 0; c < nc; ++c)
            acc += double(blk[(a * nb + b) * ncd + c * nd + r]) * __ldg(Dm + (size_t)(c0 + c) * n + b0 + b);
        atomicAdd(Km + (size_t)(a0 + a) * n + d0 + r, s * acc);
      } else {
        const int c = r - nd;
        for (int b = 0; b < nb; ++b)
          for (int d = 0; d < nd; ++d)
            acc += double(blk[(a * nb + b) * ncd + c * nd + d]) * __ldg(Dm + (size_t)(d0 + d) * n + b0 + b);
        atomicAdd(Km + (size_t)(a0 + a) * n + c0 + c, s * acc);
      }
    }
    // K[b][d] += v D[c][a]; K[b][c] += v D[d][a]
    for (int idx = lane; idx < nb * (nd + nc); idx += 32) {
      const int b = idx / (nd + nc), r = idx % (nd + nc);
      double acc = 0.0;
      if (r < nd) {
        for (int a = 0; a < na; ++a)
          for (int c = 0; c < nc; ++c)
            acc += double(blk[(a * nb + b) * ncd + c * nd + r]) * __ldg(Dm + (size_t)(c0 + c) * n + a0 + a);
        atomicAdd(Km + (size_t)(b0 + b) * n + d0 + r, s * acc);
      } else {
        const int c = r - nd;
        for (int a = 0; a < na; ++a)
          for (int d = 0; d < nd; ++d)
            acc += double(blk[(a * nb + b) * ncd + c * nd + d]) * __ldg(Dm + (size_t)(d0 + d) * n + a0 + a);
        atomicAdd(Km + (size_t)(b0 + b) * n + c0 + c, s * acc);
      }
    }
  }
}

}  // namespace jqc
