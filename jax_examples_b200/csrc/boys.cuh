// Boys function F_m(T) = int_0^1 u^{2m} exp(-T u^2) du on the device.
//
// Method (our own; the reference's boys_fn at jax_qc/integrals/boys.py:86-109
// uses upward recurrence, which is unstable for m >= 3 at small T):
//   T < 36:  F_M(T) from a table of F_m(T_i) on the grid T_i = i/16 by the
//            Taylor series  F_M(T_i - d) = sum_k F_{M+k}(T_i) d^k / k!
//            (|d| <= 1/32; 8 terms in FP64 (truncation ~2e-17 relative),
//            5 terms in FP32), then the stable downward recursion
//            F_{m-1} = (2T F_m + e^{-T}) / (2m-1), with e^{-T} from the
//            same row for M <= 2 (see kBoysDerivMaxM) and from a table of
//            e^{-T_i} above.
//   T >= 36: F_0 = sqrt(pi/T)/2 (erf(6) = 1 to 2e-17), then upward
//            recursion F_{m+1} = ((2m+1) F_m - e^{-T}) / (2T), well
//            conditioned for T > m.
// The table (kBoysRows x kBoysCols, row-major by T) is computed on the host
// in long double from the convergent series and downward recursion.
#pragma once

#include "common.cuh"

namespace jqc {

template <typename T>
struct BoysConst;
template <>
struct BoysConst<double> {
  static constexpr int kTaylor = kBoysTaylor;
};
template <>
struct BoysConst<float> {
  static constexpr int kTaylor = kBoysTaylorF;
};

__device__ __forceinline__ double boys_exp(double x) { return exp(x); }
__device__ __forceinline__ float boys_exp(float x) { return expf(x); }
__device__ __forceinline__ double boys_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float boys_sqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double boys_rsqrt(double x) { return rsqrt(x); }
__device__ __forceinline__ float boys_rsqrt(float x) { return rsqrtf(x); }
__device__ __forceinline__ int boys_round(double x) { return __double2int_rn(x); }
__device__ __forceinline__ int boys_round(float x) { return __float2int_rn(x); }

template <typename T>
struct RoundMagic;
template <>
struct RoundMagic<double> {
  static constexpr double value = 6755399441055744.0;  // 1.5 * 2^52
  static __device__ __forceinline__ int low(double x) { return __double2loint(x); }
};
template <>
struct RoundMagic<float> {
  static constexpr float value = 12582912.0f;  // 1.5 * 2^23
  static __device__ __forceinline__ int low(float x) { return __float_as_int(x) - 0x4B400000; }
};

__host__ __device__ constexpr double inv_factorial(int k) {
  double f = 1.0;
  for (int j = 2; j <= k; ++j) f *= j;
  return 1.0 / f;
}

// Aligned per-order table used by the hot kernels: for order M and grid
// point i the 8 values F_{M+k}(T_i) / k!, k < 8, are one 64-byte (FP64) or
// 32-byte (FP32) aligned row at tabA[(M * kBoysRows + i) * 8], fetched with 16-byte
// vector loads.
constexpr int kBoysARow = 8;
// After the (kBoysMaxM+1) x kBoysRows rows of the aligned table come the
// kBoysExpRows values e^{-T_i} (T_i up to kBoysExpTEnd): e^{-t} = e^{-T_i}
// e^{T_i - t} with |T_i - t| <= 1/32, so a short Taylor series replaces the
// exponential on both sides of kBoysTMax, and the lanes of a warp that fall
// on different sides of it share that part of the work.
constexpr int kBoysExpOff = (kBoysMaxM + 1) * kBoysRows * kBoysARow;
constexpr int kBoysAlignedSize = kBoysExpOff + kBoysExpRows;

// 32-byte vector loads through the read-only data path (256-bit loads,
// sm_100 and later); the address must be 32-byte aligned.  One load of a
// 32-byte record is one L1 request where two 16-byte loads were two, which
// matters for the scattered per-lane reads (table rows, primitive pairs) that
// bound the low-L kernels.
__device__ __forceinline__ void ldg32B(const double* __restrict__ p, double& a, double& b, double& c, double& d) {
  asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(a), "=d"(b), "=d"(c), "=d"(d) : "l"(p));
}
__device__ __forceinline__ void ldg32B(const float* __restrict__ p, float (&v)[8]) {
  asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7])
      : "l"(p));
}

__device__ __forceinline__ void boys_row(const double* __restrict__ r, double (&v)[8]) {
  ldg32B(r, v[0], v[1], v[2], v[3]);
  ldg32B(r + 4, v[4], v[5], v[6], v[7]);
}
__device__ __forceinline__ void boys_row(const float* __restrict__ r, float (&v)[8]) { ldg32B(r, v); }

// Orders up to this take e^{-t} of the Taylor branch from the table row
// itself: the row of order M holds F_{M+k}(T_i)/k!, so the derivative of the
// Taylor polynomial is F_{M+1}(t) (one term shorter) and
//   e^{-t} = (2M+1) F_M(t) - 2t F_{M+1}(t)
// (the upward recursion solved for e^{-t}).  The cancellation at large t
// costs nothing: the error it leaves in e^{-t} is a rounding of F_M, which the
// downward recursion divides by 2t.  Measured against 40-digit values over
// [0, 36): 4.4e-16 (M = 1) and 8.7e-16 (M = 2) largest relative error of
// F_0..F_M, against 2.2e-15 at M = 6 (the shorter F_{M+1} series), so the
// higher orders keep the tabulated e^{-T_i}.  Dropping that load from the
// Taylor lanes matters because a scattered per-lane load costs one L1
// wavefront per lane whatever its width: the table gathers bound the low-L
// J/K kernels.
constexpr int kBoysDerivMaxM = 2;

// The asymptotic branch needs e^{-t} only while it is above 2^-60 of
// (2m+1) F_m(t) for some m < M: up to t = 44, 48, 51, 54, 56, 59, 61, 64 for
// M = 1..8 (81 at M = 16); beyond 42 + 3M its term is dropped (and not loaded).
__host__ __device__ constexpr int boys_exp_tcut(int M) { return 42 + 3 * M; }

// Writes F_0 .. F_M at T into F[0..M] from the aligned table `tabA`.  For
// M <= kBoysDerivMaxM every lane issues one gather at most: the table row
// (Taylor branch) or the e^{-T_i} value (asymptotic branch below
// boys_exp_tcut).
template <typename T, int M>
__device__ __forceinline__ void boys_eval(T t, const T* __restrict__ tabA, T (&F)[M + 1]) {
  constexpr int KT = BoysConst<T>::kTaylor;
  constexpr bool kDeriv = M > 0 && M <= kBoysDerivMaxM;
  // FP32 rows carry 8 values of which F_M's series uses KT = 5; with the
  // derivative it takes one more (6 terms for F_M, 5 for F_{M+1}).  FP64 uses
  // all 8 (8 and 7).
  constexpr int KP = (kDeriv && KT < kBoysARow) ? KT + 1 : KT;
  const T tc = t < T(kBoysExpTEnd) ? t : T(kBoysExpTEnd);
  // i = round(16 tc) without conversion instructions: adding 1.5 * 2^52
  // (2^23 in FP32) to 0 <= x < 2^22 leaves round-to-nearest(x) in the low
  // mantissa bits, and subtracting it again gives that integer exactly.
  const T xr = tc * T(kBoysGridInv) + RoundMagic<T>::value;
  const int i = RoundMagic<T>::low(xr);
  const T d = (xr - RoundMagic<T>::value) * T(1.0 / kBoysGridInv) - tc;  // T_i - t, |d| <= 1/32
  const bool taylor = t < T(kBoysTMax);
  T eT = T(0);
  if constexpr (kDeriv) {
    if (!taylor && t < T(boys_exp_tcut(M))) eT = __ldg(tabA + kBoysExpOff + i);
  } else if constexpr (M > 0) {
    eT = __ldg(tabA + kBoysExpOff + i);
  }
  // e^{-t} = e^{-T_i} e^{d}, e^d by Horner over the coefficients 1/k!
  auto exp_d = [&]() {
    T ed = T(inv_factorial(KT - 1));
#pragma unroll
    for (int k = KT - 2; k >= 0; --k) ed = ed * d + T(inv_factorial(k));
    return eT * ed;
  };
  T e = T(0);
  if constexpr (M > 0 && !kDeriv) e = exp_d();
  if (taylor) {
    // the row holds F_{M+k}(T_i) / k!: the Taylor series in d is a Horner
    // chain of fused multiply-adds
    T v[8];
    boys_row(tabA + (M * kBoysRows + i) * kBoysARow, v);
    if constexpr (kDeriv) {
      // value and derivative of the polynomial in one pass
      T acc = v[KP - 1], der = T(0);
#pragma unroll
      for (int k = KP - 2; k >= 0; --k) {
        der = der * d + acc;
        acc = acc * d + v[k];
      }
      F[M] = acc;
      e = T(2 * M + 1) * acc - (t + t) * der;
    } else {
      T acc = v[KT - 1];
#pragma unroll
      for (int k = KT - 2; k >= 0; --k) acc = acc * d + v[k];
      F[M] = acc;
    }
    if constexpr (M > 0) {
      const T t2 = t + t;
#pragma unroll
      for (int m = M - 1; m >= 0; --m) F[m] = (t2 * F[m + 1] + e) * T(1.0 / (2 * m + 1));
    }
  } else {
    const T r = boys_rsqrt(t);
    F[0] = T(0.88622692545275801364908374167057) * r;  // sqrt(pi)/2 / sqrt(t)
    if constexpr (M > 0) {
      if constexpr (kDeriv) e = exp_d();
      const T half_inv_t = T(0.5) * (r * r);
#pragma unroll
      for (int m = 0; m < M; ++m) F[m + 1] = (T(2 * m + 1) * F[m] - e) * half_inv_t;
    }
  }
}

// Runtime-order variant for the standalone Boys kernel (m <= kBoysMaxM).
template <typename T>
__device__ __forceinline__ void boys_eval_rt(T t, const T* __restrict__ tab, int M, T* F) {
  constexpr int KT = BoysConst<T>::kTaylor;
  if (t < T(kBoysTMax)) {
    const int i = boys_round(t * T(kBoysGridInv));
    const T d = T(i) * T(1.0 / kBoysGridInv) - t;
    const T* row = tab + i * kBoysCols + M;
    T acc = row[KT - 1];
    for (int k = KT - 2; k >= 0; --k) acc = row[k] + acc * (d / T(k + 1));
    F[M] = acc;
    const T e = boys_exp(-t);
    for (int m = M - 1; m >= 0; --m) F[m] = (T(2) * t * F[m + 1] + e) / T(2 * m + 1);
  } else {
    const T inv_t = T(1) / t;
    F[0] = T(0.88622692545275801364908374167057) * boys_sqrt(inv_t);
    const T e = boys_exp(-t);
    for (int m = 0; m < M; ++m) F[m + 1] = (T(2 * m + 1) * F[m] - e) * T(0.5) * inv_t;
  }
}

// Host: fill the FP64 table (kBoysRows * kBoysCols) in long double.
void boys_fill_table(double* tab);

// Per-device lazily created tables (device pointers): the row-major base
// table (kBoysRows x kBoysCols) and the aligned per-order table
// ((kBoysMaxM+1) x kBoysRows x 8), FP64 and FP32.  The first call on a device
// allocates and uploads them; later calls return the cached pointers.
struct BoysTables {
  const double* t64;
  const float* t32;
  const double* a64;
  const float* a32;
};
int boys_tables(int device, const double** d64, const float** d32);
int boys_tables_all(int device, BoysTables* out);

}  // namespace jqc
