// One-electron derivative terms of the RHF gradient over shell pairs (a >= b
// in shell order):
//   grad += sum_ab D_ab d(T+V)_ab/dR - W_ab dS_ab/dR
// (the reference differentiates these integrals with JAX in
// jax_qc/grad/rhf_grad.py:92-103; here they are written out).
//
// McMurchie-Davidson with derivative E coefficients on centre A
// (2 alpha E_{i+1} - i E_{i-1}), d/dB = -d/dA for S and T, and for the
// nuclear attraction of nucleus C the operator-centre term
// dV/dC_x = -Z_C (2 pi/p) K sum E E E (-R_{t+1,u,v}) (Hellmann-Feynman) with
// dV/dB = -dV/dA - dV/dC.
//
// Both kernels take one warp per shell pair and fix the pair's angular
// momenta at compile time (one launch per (la, lb) class):
//   grad1e_st_kernel  lanes over the primitive pairs of the shell pair,
//   grad1e_v_kernel   lanes over the nuclei, the primitive pairs in a loop.
// E coefficients, the Boys values (aligned table, compile-time order) and the
// Hermite integrals stay in registers; the forces are reduced over the warp
// before the atomics.
#include "kernels.cuh"
#include "warp_engine.cuh"

namespace jqc {

namespace {

constexpr double kG1Pi = 3.14159265358979323846;

__device__ __forceinline__ bool g1_pair(int idx, int& i, int& j) {
  i = (int)((sqrt(8.0 * idx + 1.0) - 1.0) * 0.5);
  while (i * (i + 1) / 2 > idx) --i;
  while ((i + 1) * (i + 2) / 2 <= idx) ++i;
  j = idx - i * (i + 1) / 2;
  return true;
}

// E coefficients of one primitive pair along the three axes up to
// (LA + DA, LB + DB).
template <int LA, int LB>
struct G1E {
  double e[3][LA + 1][LB + 1][LA + LB + 1];
};

template <int LA, int LB>
__device__ __forceinline__ void g1_ecoef(G1E<LA, LB>& q, const double* A, const double* B, const double* P,
                                         double inv2p) {
  static_for<3>([&](auto x_) {
    constexpr int x = decltype(x_)::value;
    ecoef_compute<double, LA, LB, false>(q.e[x], P[x] - A[x], P[x] - B[x], inv2p);
  });
}

// Cartesian exponent of component k of angular momentum l along axis x.
__host__ __device__ constexpr int g1_c(int l, int k, int x) {
  return x == 0 ? cart_lx(l, k) : (x == 1 ? cart_ly(l, k) : cart_lz(l, k));
}

__device__ __forceinline__ double g1_warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// ---------------------------------------------------------------- S and T
template <int LA, int LB>
__device__ void g1_st_pair(const Grad1Params& p, int i, int j, int lane) {
  constexpr int NA = ncart(LA), NB = ncart(LB);
  const double* A = p.centres + 3 * i;
  const double* B = p.centres + 3 * j;
  const int a0 = p.ao[i], b0 = p.ao[j];
  const double ab2 = (A[0] - B[0]) * (A[0] - B[0]) + (A[1] - B[1]) * (A[1] - B[1]) + (A[2] - B[2]) * (A[2] - B[2]);
  const int na = p.nprim[i], nb = p.nprim[j];
  double gA[3] = {0.0, 0.0, 0.0};
  for (int k = lane; k < na * nb; k += 32) {
    const int ia = k / nb, ib = k - (k / nb) * nb;
    const double al = p.exps[p.prim_off[i] + ia], be = p.exps[p.prim_off[j] + ib];
    const double pp = al + be;
    const double P[3] = {(al * A[0] + be * B[0]) / pp, (al * A[1] + be * B[1]) / pp, (al * A[2] + be * B[2]) / pp};
    const double K = exp(-(al * be / pp) * ab2) * p.coefs[p.prim_off[i] + ia] * p.coefs[p.prim_off[j] + ib];
    G1E<LA + 2, LB + 1> q;
    g1_ecoef<LA + 2, LB + 1>(q, A, B, P, 0.5 / pp);
    const double sq = sqrt(kG1Pi / pp);
    // 1-D overlaps S1[x][a][b] = sqrt(pi/p) E_0 and kinetic T1 of the reference's
    // formula, a <= LA + 1 (the A derivative), b <= LB
    double S1[3][LA + 3][LB + 2], T1[3][LA + 2][LB + 1];
    static_for<3>([&](auto x_) {
      constexpr int x = decltype(x_)::value;
      static_for<LA + 3>([&](auto a_) {
        constexpr int a = decltype(a_)::value;
        static_for<LB + 2>([&](auto b_) {
          constexpr int b = decltype(b_)::value;
          S1[x][a][b] = sq * q.e[x][a][b][0];
        });
      });
      static_for<LA + 2>([&](auto a_) {
        constexpr int a = decltype(a_)::value;
        static_for<LB + 1>([&](auto b_) {
          constexpr int b = decltype(b_)::value;
          double tv = 4.0 * al * be * S1[x][a + 1][b + 1];
          if constexpr (a > 0 && b > 0) tv += double(a * b) * S1[x][a - 1][b - 1];
          if constexpr (b > 0) tv -= 2.0 * al * b * S1[x][a + 1][b - 1];
          if constexpr (a > 0) tv -= 2.0 * be * a * S1[x][a - 1][b + 1];
          T1[x][a][b] = 0.5 * tv;
        });
      });
    });
    static_for<NA * NB>([&](auto ab_) {
      constexpr int ab = decltype(ab_)::value, ia_ = ab / NB, ib_ = ab % NB;
      const double dv = __ldg(p.D + (size_t)(a0 + ia_) * p.n + b0 + ib_);
      const double wv = __ldg(p.W + (size_t)(a0 + ia_) * p.n + b0 + ib_);
      double s[3], tk[3], ds[3], dt[3];
      static_for<3>([&](auto x_) {
        constexpr int x = decltype(x_)::value;
        constexpr int ax = g1_c(LA, ia_, x), bx = g1_c(LB, ib_, x);
        s[x] = S1[x][ax][bx];
        tk[x] = T1[x][ax][bx];
        ds[x] = 2.0 * al * S1[x][ax + 1][bx];
        dt[x] = 2.0 * al * T1[x][ax + 1][bx];
        if constexpr (ax > 0) {
          ds[x] -= ax * S1[x][ax - 1][bx];
          dt[x] -= ax * T1[x][ax - 1][bx];
        }
      });
      static_for<3>([&](auto x_) {
        constexpr int x = decltype(x_)::value, y = (x + 1) % 3, z = (x + 2) % 3;
        const double dS = ds[x] * s[y] * s[z];
        const double dT = dt[x] * s[y] * s[z] + ds[x] * (tk[y] * s[z] + s[y] * tk[z]);
        gA[x] += K * (dv * dT - wv * dS);
      });
    });
  }
  const double fac = (i == j) ? 1.0 : 2.0;
  static_for<3>([&](auto x_) {
    constexpr int x = decltype(x_)::value;
    const double v = g1_warp_sum(gA[x]) * fac;
    if (lane == 0) {
      atomicAdd(p.grad + 3 * p.atom[i] + x, v);
      atomicAdd(p.grad + 3 * p.atom[j] + x, -v);
    }
  });
}

// -------------------------------------------------------- nuclear attraction
constexpr int kG1Warps = 4;

// The E coefficients depend only on the primitive pair, the same for every
// lane (nucleus) of the warp: lanes 0..2 build one axis each in warp-shared
// memory and every lane reads them there, so a thread holds only R, the
// density block and its sums.
template <int LA, int LB>
__device__ void g1_v_pair(const Grad1Params& p, int i, int j, int lane) {
  constexpr int NA = ncart(LA), NB = ncart(LB);
  constexpr int L = LA + LB + 1;
  __shared__ double sE[kG1Warps][3][LA + 2][LB + 1][LA + LB + 2];
  double (*E)[LA + 2][LB + 1][LA + LB + 2] = sE[threadIdx.x >> 5];
  const double* A = p.centres + 3 * i;
  const double* B = p.centres + 3 * j;
  const int a0 = p.ao[i], b0 = p.ao[j];
  const double ab2 = (A[0] - B[0]) * (A[0] - B[0]) + (A[1] - B[1]) * (A[1] - B[1]) + (A[2] - B[2]) * (A[2] - B[2]);
  const int mol = p.shell_mol ? p.shell_mol[i] : -1;
  double dab[NA * NB];
  static_for<NA * NB>([&](auto ab_) {
    constexpr int ab = decltype(ab_)::value;
    dab[ab] = __ldg(p.D + (size_t)(a0 + ab / NB) * p.n + b0 + ab % NB);
  });
  const int na = p.nprim[i], nb = p.nprim[j];
  double gAsum[3] = {0.0, 0.0, 0.0}, gBsum[3] = {0.0, 0.0, 0.0};
  for (int c0 = 0; c0 < p.n_atom; c0 += 32) {
    const int c = c0 + lane;
    const bool act = c < p.n_atom && (mol < 0 || p.atom_mol[c] == mol);
    double gA[3] = {0.0, 0.0, 0.0}, gC[3] = {0.0, 0.0, 0.0};
    const int cc = act ? c : 0;
    const double Cx = p.atom_xyz[3 * cc], Cy = p.atom_xyz[3 * cc + 1], Cz = p.atom_xyz[3 * cc + 2];
    const double Zc = p.atom_Z[cc];
    for (int ia = 0; ia < na; ++ia)
      for (int ib = 0; ib < nb; ++ib) {
        const double al = p.exps[p.prim_off[i] + ia], be = p.exps[p.prim_off[j] + ib];
        const double pp = al + be;
        const double Px = (al * A[0] + be * B[0]) / pp, Py = (al * A[1] + be * B[1]) / pp,
                     Pz = (al * A[2] + be * B[2]) / pp;
        __syncwarp();  // every lane is done with the previous primitive pair's E
        if (lane < 3) {
          const double Pl = lane == 0 ? Px : (lane == 1 ? Py : Pz);
          ecoef_compute<double, LA + 1, LB, false>(E[lane], Pl - A[lane], Pl - B[lane], 0.5 / pp);
        }
        __syncwarp();
        if (!act) continue;
        const double K = exp(-(al * be / pp) * ab2) * p.coefs[p.prim_off[i] + ia] * p.coefs[p.prim_off[j] + ib];
        const double X = Px - Cx, Y = Py - Cy, Z = Pz - Cz;
        double F[L + 1];
        boys_eval<double, L>(pp * (X * X + Y * Y + Z * Z), p.boys_al, F);
        double Rn[L + 1];
        double pw = -Zc * (2.0 * kG1Pi / pp) * K;
        static_for<L + 1>([&](auto m_) {
          constexpr int m = decltype(m_)::value;
          Rn[m] = pw * F[m];
          pw *= -2.0 * pp;
        });
        double R[nherm(L)];
        hermite_R<double, L>(R, Rn, X, Y, Z);
        static_for<NA * NB>([&](auto ab_) {
          constexpr int ab = decltype(ab_)::value, ia_ = ab / NB, ib_ = ab % NB;
          const double dv = dab[ab];
          static_for<3>([&](auto x_) {
            constexpr int x = decltype(x_)::value, y = (x + 1) % 3, z = (x + 2) % 3;
            constexpr int ax = g1_c(LA, ia_, x), bx = g1_c(LB, ib_, x);
            constexpr int ay = g1_c(LA, ia_, y), by = g1_c(LB, ib_, y);
            constexpr int az = g1_c(LA, ia_, z), bz = g1_c(LB, ib_, z);
            double accA = 0.0, accC = 0.0;
            static_for<ax + bx + 2>([&](auto t_) {
              constexpr int t = decltype(t_)::value;
              double de = 2.0 * al * E[x][ax + 1][bx][t];
              if constexpr (ax > 0 && t <= ax - 1 + bx) de -= ax * E[x][ax - 1][bx][t];
              static_for<ay + by + 1>([&](auto u_) {
                constexpr int u = decltype(u_)::value;
                static_for<az + bz + 1>([&](auto v_) {
                  constexpr int v = decltype(v_)::value;
                  constexpr int h0 = x == 0 ? t : (y == 0 ? u : v);
                  constexpr int h1 = x == 1 ? t : (y == 1 ? u : v);
                  constexpr int h2 = x == 2 ? t : (y == 2 ? u : v);
                  const double eyz = E[y][ay][by][u] * E[z][az][bz][v];
                  accA += de * eyz * R[herm_index(h0, h1, h2)];
                  if constexpr (t <= ax + bx) {
                    constexpr int k0 = h0 + (x == 0), k1 = h1 + (x == 1), k2 = h2 + (x == 2);
                    accC -= E[x][ax][bx][t] * eyz * R[herm_index(k0, k1, k2)];
                  }
                });
              });
            });
            gA[x] += dv * accA;
            gC[x] += dv * accC;
          });
        });
      }
    const double fac = (i == j) ? 1.0 : 2.0;
    static_for<3>([&](auto x_) {
      constexpr int x = decltype(x_)::value;
      if (act) atomicAdd(p.grad + 3 * c + x, fac * gC[x]);
      gAsum[x] += fac * gA[x];
      gBsum[x] -= fac * (gA[x] + gC[x]);
    });
  }
  static_for<3>([&](auto x_) {
    constexpr int x = decltype(x_)::value;
    const double va = g1_warp_sum(gAsum[x]), vb = g1_warp_sum(gBsum[x]);
    if (lane == 0) {
      atomicAdd(p.grad + 3 * p.atom[i] + x, va);
      atomicAdd(p.grad + 3 * p.atom[j] + x, vb);
    }
  });
}


}  // namespace

// One kernel per (la, lb) shell-pair class, so each gets its own register
// allocation; a warp whose pair is of another class returns at once.
template <int LA, int LB>
__global__ void __launch_bounds__(32 * kG1Warps) grad1e_st_kernel(const Grad1Params p) {
  const int idx = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (idx >= p.n_shell * (p.n_shell + 1) / 2) return;
  int i, j;
  g1_pair(idx, i, j);
  if (p.l[i] != LA || p.l[j] != LB) return;
  if (p.shell_mol && p.shell_mol[i] != p.shell_mol[j]) return;  // shells of two molecules of a batch
  g1_st_pair<LA, LB>(p, i, j, lane);
}

template <int LA, int LB>
__global__ void __launch_bounds__(32 * kG1Warps) grad1e_v_kernel(const Grad1Params p) {
  const int idx = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (idx >= p.n_shell * (p.n_shell + 1) / 2) return;
  int i, j;
  g1_pair(idx, i, j);
  if (p.l[i] != LA || p.l[j] != LB) return;
  if (p.shell_mol && p.shell_mol[i] != p.shell_mol[j]) return;
  g1_v_pair<LA, LB>(p, i, j, lane);
}

template <int LA, int LB>
static void g1_launch(const Grad1Params& p, unsigned grid, cudaStream_t s) {
  grad1e_st_kernel<LA, LB><<<grid, 32 * kG1Warps, 0, s>>>(p);
  if (p.n_atom > 0) grad1e_v_kernel<LA, LB><<<grid, 32 * kG1Warps, 0, s>>>(p);
}

cudaError_t launch_grad1e(const Grad1Params& p, cudaStream_t s) {
  const long long npair = (long long)p.n_shell * (p.n_shell + 1) / 2;
  if (npair == 0) return cudaSuccess;
  if (p.l == nullptr || p.boys_al == nullptr) return cudaErrorInvalidValue;
  const unsigned grid = (unsigned)((npair + kG1Warps - 1) / kG1Warps);
  g1_launch<0, 0>(p, grid, s);
  g1_launch<0, 1>(p, grid, s);
  g1_launch<0, 2>(p, grid, s);
  g1_launch<1, 0>(p, grid, s);
  g1_launch<1, 1>(p, grid, s);
  g1_launch<1, 2>(p, grid, s);
  g1_launch<2, 0>(p, grid, s);
  g1_launch<2, 1>(p, grid, s);
  g1_launch<2, 2>(p, grid, s);
  return cudaGetLastError();
}

}  // namespace jqc
