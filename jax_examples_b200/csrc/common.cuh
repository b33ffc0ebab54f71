// Shared definitions of the two-electron library (libjqc.so, sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <utility>

#include "../../include/jqc.h"

namespace jqc {

// Highest shell angular momentum the kernels take (Cartesian s, p, d).
constexpr int kMaxL = 2;
// Highest Boys order used anywhere: (dd|dd) gradients need L = 9; the table
// covers up to kBoysMaxM for the standalone Boys entry point.
constexpr int kBoysMaxM = 16;

// Boys table: F_m(T_i), T_i = i / kBoysGridInv, m = 0 .. kBoysCols-1.
constexpr int kBoysGridInv = 16;          // grid step 1/16
constexpr double kBoysTMax = 36.0;        // table range [0, 36); asymptotic above
constexpr int kBoysRows = 36 * kBoysGridInv + 1;
constexpr int kBoysTaylor = 8;            // Taylor terms (|dT| <= 1/32 -> ~2e-17 rel)
constexpr int kBoysTaylorF = 5;           // FP32 Taylor terms
constexpr int kBoysCols = kBoysMaxM + kBoysTaylor + 1;
// The values e^{-T_i} for the Boys recursions continue the grid to T = 746,
// where e^{-T} underflows to 0 in FP64 (and long before in FP32).
constexpr int kBoysExpTEnd = 746;
constexpr int kBoysExpRows = kBoysExpTEnd * kBoysGridInv + 1;

void set_error(const std::string& msg);

#define JQC_CUDA_CHECK(expr)                                                      \
  do {                                                                            \
    cudaError_t _e = (expr);                                                      \
    if (_e != cudaSuccess) {                                                      \
      ::jqc::set_error(std::string(#expr) + ": " + cudaGetErrorString(_e));       \
      (void)cudaGetLastError(); /* reported here: not again by a later launch */ \
      return JQC_ERR_CUDA;                                                        \
    }                                                                             \
  } while (0)

__host__ __device__ constexpr int ncart(int l) { return (l + 1) * (l + 2) / 2; }
__host__ __device__ constexpr int nherm(int L) { return (L + 1) * (L + 2) * (L + 3) / 6; }

// Cartesian component k of angular momentum l in libint order (lx descending,
// then ly descending), as jax_qc/integrals/mcmurchie_davidson.py:39-50.
__host__ __device__ constexpr int cart_lx(int l, int k) {
  int lx = l;
  while (k > l - lx) { k -= (l - lx + 1); --lx; }
  return lx;
}
__host__ __device__ constexpr int cart_ly(int l, int k) {
  int lx = l;
  while (k > l - lx) { k -= (l - lx + 1); --lx; }
  return (l - lx) - k;
}
__host__ __device__ constexpr int cart_lz(int l, int k) { return l - cart_lx(l, k) - cart_ly(l, k); }

// Index of Hermite (t,u,v) in a shell-by-total-order layout:
// all s = t+u+v < current first, then libint order within s.
__host__ __device__ constexpr int herm_index(int t, int u, int v) {
  int s = t + u + v;
  return s * (s + 1) * (s + 2) / 6 + (s - t) * (s - t + 1) / 2 + (s - t - u);
}

// Compile-time loop: f(std::integral_constant<int, i>{}) for i = 0..N-1,
// fully expanded by the front end (no reliance on the loop unroller).
template <typename F, int... Is>
__host__ __device__ __forceinline__ void static_for_impl(F&& f, std::integer_sequence<int, Is...>) {
  (f(std::integral_constant<int, Is>{}), ...);
}
template <int N, typename F>
__host__ __device__ __forceinline__ void static_for(F&& f) {
  if constexpr (N > 0) static_for_impl(f, std::make_integer_sequence<int, N>{});
}

}  // namespace jqc
