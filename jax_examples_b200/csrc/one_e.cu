// One-electron matrices S, T, V over Cartesian shells on the device.
//
// Same McMurchie-Davidson formulas as the reference
// (jax_qc/integrals/obara_saika.py:69-222):
//   S_ij (1-D) = sqrt(pi/p) E^{ij}_0
//   T_ij (1-D) = 1/2 [4 a b S_{i+1,j+1} + i j S_{i-1,j-1} - 2 a j S_{i+1,j-1}
//                     - 2 b i S_{i-1,j+1}]
//   S = K Sx Sy Sz,  T = K (Tx Sy Sz + Sx Ty Sz + Sx Sy Tz)
//   V = -sum_C Z_C (2 pi / p) K sum_tuv E_t E_u E_v R_tuv(p, P - C)
// One thread per shell pair (a >= b in shell order) and all its primitive
// pairs; the block is written to (a,b) and its transpose to (b,a).  This is
// N^2 work and far from the hot path.
#include "kernels.cuh"
#include "warp_engine.cuh"

namespace jqc {

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

// One warp per shell pair: the lanes split the nuclei of V; lane 0 adds the
// overlap and kinetic terms; the three blocks are reduced over the warp.
__global__ void one_e_kernel(const OneEParams p) {
  const int idx = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  const int npair = p.n_shell * (p.n_shell + 1) / 2;
  if (idx >= npair) return;
  int i = (int)((sqrt(8.0 * idx + 1.0) - 1.0) * 0.5);
  while (i * (i + 1) / 2 > idx) --i;
  while ((i + 1) * (i + 2) / 2 <= idx) ++i;
  const int j = idx - i * (i + 1) / 2;
  const int la = p.l[i], lb = p.l[j];
  const int na = ncart(la), nb = ncart(lb);
  const double* A = p.centres + 3 * i;
  const double* B = p.centres + 3 * j;
  double s[36], t[36], v[36];
  for (int x = 0; x < na * nb; ++x) s[x] = t[x] = v[x] = 0.0;
  const double ab2 = (A[0] - B[0]) * (A[0] - B[0]) + (A[1] - B[1]) * (A[1] - B[1]) + (A[2] - B[2]) * (A[2] - B[2]);
  // shells of different molecules of a batch: the block stays zero
  const int mol = p.shell_mol ? p.shell_mol[i] : 0;
  const int npa = (p.shell_mol && p.shell_mol[j] != mol) ? 0 : p.nprim[i];
  for (int ia = 0; ia < npa; ++ia)
    for (int ib = 0; ib < p.nprim[j]; ++ib) {
      const double al = p.exps[p.prim_off[i] + ia], be = p.exps[p.prim_off[j] + ib];
      const double w = p.coefs[p.prim_off[i] + ia] * p.coefs[p.prim_off[j] + ib];
      const double pp = al + be;
      const double P[3] = {(al * A[0] + be * B[0]) / pp, (al * A[1] + be * B[1]) / pp, (al * A[2] + be * B[2]) / pp};
      const double K = exp(-(al * be / pp) * ab2) * w;
      const double inv2p = 0.5 / pp;
      // extended E (for kinetic) up to (la+1, lb+1): dims [4][4][7]
      double E[3][4][4][7];
      double S1[3][4][4], T1[3][3][3];
      for (int x = 0; x < 3; ++x) {
        const double pa = P[x] - A[x], pb = P[x] - B[x];
        for (int a = 0; a <= la + 1; ++a)
          for (int b = 0; b <= lb + 1; ++b)
            for (int tt = 0; tt < 7; ++tt) E[x][a][b][tt] = 0.0;
        E[x][0][0][0] = 1.0;
        for (int a = 0; a < la + 1; ++a)
          for (int tt = 0; tt <= a + 1; ++tt) {
            double val = 0.0;
            if (tt <= a) val = pa * E[x][a][0][tt];
            if (tt >= 1) val += inv2p * E[x][a][0][tt - 1];
            if (tt + 1 <= a) val += (tt + 1) * E[x][a][0][tt + 1];
            E[x][a + 1][0][tt] = val;
          }
        for (int b = 0; b < lb + 1; ++b)
          for (int a = 0; a <= la + 1; ++a)
            for (int tt = 0; tt <= a + b + 1; ++tt) {
              double val = 0.0;
              if (tt <= a + b) val = pb * E[x][a][b][tt];
              if (tt >= 1) val += inv2p * E[x][a][b][tt - 1];
              if (tt + 1 <= a + b) val += (tt + 1) * E[x][a][b][tt + 1];
              E[x][a][b + 1][tt] = val;
            }
        const double sq = sqrt(M_PI / pp);
        for (int a = 0; a <= la + 1; ++a)
          for (int b = 0; b <= lb + 1; ++b) S1[x][a][b] = sq * E[x][a][b][0];
        for (int a = 0; a <= la; ++a)
          for (int b = 0; b <= lb; ++b) {
            double tv = 4.0 * al * be * S1[x][a + 1][b + 1];
            if (a > 0 && b > 0) tv += a * b * S1[x][a - 1][b - 1];
            if (b > 0) tv -= 2.0 * al * b * S1[x][a + 1][b - 1];
            if (a > 0) tv -= 2.0 * be * a * S1[x][a - 1][b + 1];
            T1[x][a][b] = 0.5 * tv;
          }
      }
      if (lane == 0)
        for (int a = 0; a < na; ++a)
          for (int b = 0; b < nb; ++b) {
            int ax, ay, az, bx, by, bz;
            wcart(la, a, ax, ay, az);
            wcart(lb, b, bx, by, bz);
            const double sx = S1[0][ax][bx], sy = S1[1][ay][by], sz = S1[2][az][bz];
            s[a * nb + b] += K * sx * sy * sz;
            t[a * nb + b] += K * (T1[0][ax][bx] * sy * sz + sx * T1[1][ay][by] * sz + sx * sy * T1[2][az][bz]);
          }
      // nuclear attraction, nuclei split over the lanes
      const int L = la + lb;
      for (int c = lane; c < p.n_atom; c += 32) {
        if (p.atom_mol && p.atom_mol[c] != mol) continue;  // nuclei of this molecule only
        const double X = P[0] - p.atom_xyz[3 * c], Y = P[1] - p.atom_xyz[3 * c + 1], Z = P[2] - p.atom_xyz[3 * c + 2];
        double F[kBoysMaxM + 1];
        boys_eval_rt<double>(pp * (X * X + Y * Y + Z * Z), p.boys, L, F);
        const double pref = -p.atom_Z[c] * (2.0 * M_PI / pp) * K;
        double R[nherm(4)];
        double Rn[5];
        double pw = pref;
        for (int m = 0; m <= L; ++m) {
          Rn[m] = pw * F[m];
          pw *= -2.0 * pp;
        }
        R[0] = Rn[L];
        for (int m = L - 1; m >= 0; --m) {
          for (int sh = L - m; sh >= 1; --sh) {
            const int base = sh * (sh + 1) * (sh + 2) / 6;
            for (int k = 0; k < ncart(sh); ++k) {
              int tt, u, vv;
              wcart(sh, k, tt, u, vv);
              double val;
              if (tt > 0) {
                val = X * R[herm_index(tt - 1, u, vv)];
                if (tt > 1) val += (tt - 1) * R[herm_index(tt - 2, u, vv)];
              } else if (u > 0) {
                val = Y * R[herm_index(tt, u - 1, vv)];
                if (u > 1) val += (u - 1) * R[herm_index(tt, u - 2, vv)];
              } else {
                val = Z * R[herm_index(tt, u, vv - 1)];
                if (vv > 1) val += (vv - 1) * R[herm_index(tt, u, vv - 2)];
              }
              R[base + k] = val;
            }
          }
          R[0] = Rn[m];
        }
        for (int a = 0; a < na; ++a)
          for (int b = 0; b < nb; ++b) {
            int ax, ay, az, bx, by, bz;
            wcart(la, a, ax, ay, az);
            wcart(lb, b, bx, by, bz);
            double acc = 0.0;
            for (int t0 = 0; t0 <= ax + bx; ++t0)
              for (int u0 = 0; u0 <= ay + by; ++u0)
                for (int v0 = 0; v0 <= az + bz; ++v0)
                  acc += E[0][ax][bx][t0] * E[1][ay][by][u0] * E[2][az][bz][v0] * R[herm_index(t0, u0, v0)];
            v[a * nb + b] += acc;
          }
      }
    }
  for (int x = 0; x < na * nb; ++x) {
    double vx = v[x];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) vx += __shfl_xor_sync(0xffffffffu, vx, o);
    v[x] = vx;
  }
  if (lane != 0) return;
  const int a0 = p.ao[i], b0 = p.ao[j];
  for (int a = 0; a < na; ++a)
    for (int b = 0; b < nb; ++b) {
      const size_t r = a0 + a, c = b0 + b;
      p.S[r * p.n + c] = p.S[c * p.n + r] = s[a * nb + b];
      p.T[r * p.n + c] = p.T[c * p.n + r] = t[a * nb + b];
      p.V[r * p.n + c] = p.V[c * p.n + r] = v[a * nb + b];
    }
}

cudaError_t launch_one_e(const OneEParams& p, cudaStream_t s) {
  const long long npair = (long long)p.n_shell * (p.n_shell + 1) / 2;
  if (npair == 0) return cudaSuccess;
  one_e_kernel<<<(unsigned)((npair * 32 + 127) / 128), 128, 0, s>>>(p);
  return cudaGetLastError();
}

}  // namespace jqc
