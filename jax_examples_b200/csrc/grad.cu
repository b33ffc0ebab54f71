// Nuclear-gradient kernels: the ERI-derivative adjoint and the one-electron
// derivative terms.
//
// Two-electron part.  With Gamma_abcd = j D^t_ab D^t_cd
//     - (k/2) sum_s (D^s_ac D^s_bd + D^s_ad D^s_bc)   (D^t = sum_s D^s)
// the two-electron energy is E2 = 1/2 sum Gamma (ab|cd) and its nuclear
// gradient 1/2 sum Gamma d(ab|cd)/dR.  RHF: one density, j = 1, k = 1/2,
// which is the contraction rhf_grad.py:201-209 forms from finite differences
// (1/2 sum D (dJ - dK/2)); UHF: alpha and beta densities, j = k = 1.  Over
// canonical shell quartets that is 4 s sum_elements Gamma d(ab|cd)/dR with the
// usual 1/2 per coincidence in s.
//
// The derivative integrals are never stored.  Per primitive quartet:
//   d/dA_x phi_a = 2 alpha phi_{a+1x} - a_x phi_{a-1x}
// enters as derivative E coefficients DA^x_{ij,t} = 2 alpha E_{i+1,j,t} -
// i E_{i-1,j,t} (likewise DB with beta on the bra's second centre and DC with
// gamma on the ket's first centre), contracted with the same R_tuv and the
// ket/bra E coefficients as the integrals themselves; dD follows from
// translational invariance, dD = -(dA + dB + dC).  The bra derivatives use
// X_cd[tuv] (ket contracted against R) up to one higher bra Hermite order,
// the ket derivative a second pass of stage 1 with DC.
//
// This file holds the warp-cooperative version (runtime class, one warp per
// shell quartet, R/E/X/Gamma in shared memory); it serves every class.
#include "kernels.cuh"
#include "warp_engine.cuh"

namespace jqc {

constexpr int kGMaxL = 9;  // (dd|dd) + 1
constexpr int kGradWarps = 4;  // warps per block of the warp-cooperative gradient

// Shared-memory layout of one warp, sized for its class (la lb | lc ld):
//   Eb[3][la+2][lb+2][la+lb+3]   bra E up to one order higher
//   DA, DB[3][la+1][lb+1][la+lb+2] derivative E on the bra centres
//   Fk[3][lc+2][ld+1][lc+ld+2]   ket E with (-1)^t
//   DC[3][lc+1][ld+1][lc+ld+2]   derivative ket E on centre C
//   Rn[L+2], R[nherm(L+1)], X[ncd * nherm(la+lb+1)], G[nab * ncd]
struct GradLayout {
  int ebJ, ebT, ebX, daJ, daT, daX, fkD, fkT, fkX, dcX;
  int oDA, oDB, oFk, oDC, oRn, oR, oX, oG, total;
  __host__ __device__ GradLayout(int la, int lb, int lc, int ld) {
    ebJ = lb + 2;
    ebT = la + lb + 3;
    ebX = (la + 2) * ebJ * ebT;
    daJ = lb + 1;
    daT = la + lb + 2;
    daX = (la + 1) * daJ * daT;
    fkD = ld + 1;
    fkT = lc + ld + 2;
    fkX = (lc + 2) * fkD * fkT;
    dcX = (lc + 1) * fkD * fkT;
    const int L = la + lb + lc + ld;
    const int ncd = ncart(lc) * ncart(ld), nab = ncart(la) * ncart(lb);
    oDA = 3 * ebX;
    oDB = oDA + 3 * daX;
    oFk = oDB + 3 * daX;
    oDC = oFk + 3 * fkX;
    oRn = oDC + 3 * dcX;
    oR = oRn + L + 2;
    oX = oR + nherm(L + 1);
    oG = oX + ncd * nherm(la + lb + 1);
    total = oG + nab * ncd;
    total = (total + 1) & ~1;  // keep every warp's slice 16-byte aligned
  }
};

// E coefficients (runtime la, lb) along one axis into e[i][j][t] for
// i <= la, j <= lb, with capacity [4][4][7].
__device__ void gecoef(double (*e)[4][7], int la, int lb, double pa, double pb, double inv2p) {
  for (int i = 0; i <= la; ++i)
    for (int j = 0; j <= lb; ++j)
      for (int t = 0; t < 7; ++t) e[i][j][t] = 0.0;
  e[0][0][0] = 1.0;
  for (int i = 0; i < la; ++i)
    for (int t = 0; t <= i + 1; ++t) {
      double v = 0.0;
      if (t <= i) v = pa * e[i][0][t];
      if (t >= 1) v += inv2p * e[i][0][t - 1];
      if (t + 1 <= i) v += (t + 1) * e[i][0][t + 1];
      e[i + 1][0][t] = v;
    }
  for (int j = 0; j < lb; ++j)
    for (int i = 0; i <= la; ++i)
      for (int t = 0; t <= i + j + 1; ++t) {
        double v = 0.0;
        if (t <= i + j) v = pb * e[i][j][t];
        if (t >= 1) v += inv2p * e[i][j][t - 1];
        if (t + 1 <= i + j) v += (t + 1) * e[i][j][t + 1];
        e[i][j + 1][t] = v;
      }
}

// One warp per task (a bra primitive range of one shell quartet, or of up to
// nket quartets of one bra), kGradWarps warps per block, each with its own
// slice of the dynamic shared memory.
__global__ void __launch_bounds__(32 * kGradWarps, 4) warp_grad_kernel(const GradParams prm, int la, int lb, int lc,
                                                                   int ld) {
  extern __shared__ __align__(16) double smd[];
  const GradLayout ly(la, lb, lc, ld);
  const int lane = threadIdx.x & 31;
  const int task_id = blockIdx.x * kGradWarps + (threadIdx.x >> 5);
  if (task_id >= prm.n_tasks) return;
  double* base = smd + (size_t)(threadIdx.x >> 5) * ly.total;
  double* const sEb = base;
  double* const sDA = base + ly.oDA;
  double* const sDB = base + ly.oDB;
  double* const sFk = base + ly.oFk;
  double* const sDC = base + ly.oDC;
  double* const sRn = base + ly.oRn;
  double* const sR = base + ly.oR;
  double* const sX = base + ly.oX;
  double* const sG = base + ly.oG;
  auto EB = [&](int x, int i, int j, int t) -> double& { return sEb[x * ly.ebX + (i * ly.ebJ + j) * ly.ebT + t]; };
  auto DA = [&](int x, int i, int j, int t) -> double& { return sDA[x * ly.daX + (i * ly.daJ + j) * ly.daT + t]; };
  auto DB = [&](int x, int i, int j, int t) -> double& { return sDB[x * ly.daX + (i * ly.daJ + j) * ly.daT + t]; };
  auto FK = [&](int x, int c, int d, int t) -> double& { return sFk[x * ly.fkX + (c * ly.fkD + d) * ly.fkT + t]; };
  auto DC = [&](int x, int c, int d, int t) -> double& { return sDC[x * ly.dcX + (c * ly.fkD + d) * ly.fkT + t]; };

  const Task task = prm.tasks[task_id];
  const ShellPair bp = prm.pairs[task.bra];
  const int na = ncart(la), nb = ncart(lb), nc = ncart(lc), nd = ncart(ld);
  const int nab = na * nb, ncd = nc * nd, ntot = nab * ncd;
  const int lab = la + lb, L = la + lb + lc + ld;
  const int nh1 = nherm(lab + 1), nh0 = nherm(lab);
  const int n = prm.n;
  const double* ctr = prm.centres;
  const double Ax = ctr[3 * bp.a], Ay = ctr[3 * bp.a + 1], Az = ctr[3 * bp.a + 2];
  const double Bx = ctr[3 * bp.b], By = ctr[3 * bp.b + 1], Bz = ctr[3 * bp.b + 2];
  const int a0 = prm.ao[bp.a], b0 = prm.ao[bp.b];

  for (int kk = 0; kk < task.nket; ++kk) {
    const int kidx = task.ket0 + kk;
    const ShellPair kp = prm.pairs[kidx];
    const double Cx = ctr[3 * kp.a], Cy = ctr[3 * kp.a + 1], Cz = ctr[3 * kp.a + 2];
    const double Dx = ctr[3 * kp.b], Dy = ctr[3 * kp.b + 1], Dz = ctr[3 * kp.b + 2];
    const int c0 = prm.ao[kp.a], d0 = prm.ao[kp.b];
    // density screening (warp-uniform: one quartet at a time)
    if (prm.dmax_top != nullptr && float(bp.Q) * float(kp.Q) * gamma_bound_top(prm, *prm.dmax_top) < prm.dens_tau)
      continue;
    if (prm.dmax != nullptr && float(bp.Q) * float(kp.Q) * gamma_bound(prm, bp.a, bp.b, kp.a, kp.b) < prm.dens_tau)
      continue;
    // Gamma for this quartet
    __syncwarp();
    for (int e = lane; e < ntot; e += 32) {
      const int ab = e / ncd, cd = e % ncd;
      const int ia = a0 + ab / nb, ib = b0 + ab % nb, ic = c0 + cd / nd, id = d0 + cd % nd;
      double dab = 0.0, dcd = 0.0, kx = 0.0;
      for (int s = 0; s < prm.n_dens; ++s) {
        const double* Ds = prm.D + (size_t)s * n * n;
        dab += Ds[(size_t)ia * n + ib];
        dcd += Ds[(size_t)ic * n + id];
        kx += Ds[(size_t)ia * n + ic] * Ds[(size_t)ib * n + id] + Ds[(size_t)ia * n + id] * Ds[(size_t)ib * n + ic];
      }
      sG[e] = prm.jscale * dab * dcd - 0.5 * prm.kscale * kx;
    }
    double g[9];
    for (int k = 0; k < 9; ++k) g[k] = 0.0;

    const int p0 = task.flags & 0xffff, p1 = task.flags >> 16;  // bra primitive-pair range
    for (int ip = p0; ip < p1; ++ip) {
      const PrimPair bpp = prm.pp[bp.pp + ip];
      __syncwarp();
      if (lane < 3) {
        const double P = lane == 0 ? bpp.Px : lane == 1 ? bpp.Py : bpp.Pz;
        const double A = lane == 0 ? Ax : lane == 1 ? Ay : Az;
        const double B = lane == 0 ? Bx : lane == 1 ? By : Bz;
        double E[4][4][7];
        gecoef(E, la + 1, lb + 1, P - A, P - B, bpp.h);
        for (int i = 0; i <= la + 1; ++i)
          for (int j = 0; j <= lb + 1; ++j)
            for (int t = 0; t < ly.ebT; ++t) EB(lane, i, j, t) = E[i][j][t];
        for (int i = 0; i <= la; ++i)
          for (int j = 0; j <= lb; ++j)
            for (int t = 0; t <= la + lb + 1; ++t) {
              double va = 2.0 * bpp.alpha * E[i + 1][j][t];
              if (i > 0) va -= i * E[i - 1][j][t];
              double vb = 2.0 * bpp.beta * E[i][j + 1][t];
              if (j > 0) vb -= j * E[i][j - 1][t];
              DA(lane, i, j, t) = va;
              DB(lane, i, j, t) = vb;
            }
      }
      for (int iq = 0; iq < kp.npp; ++iq) {
        const PrimPair kpp = prm.pp[kp.pp + iq];
        if (lane >= 3 && lane < 6) {
          const int ax = lane - 3;
          const double Q = ax == 0 ? kpp.Px : ax == 1 ? kpp.Py : kpp.Pz;
          const double C = ax == 0 ? Cx : ax == 1 ? Cy : Cz;
          const double Dd = ax == 0 ? Dx : ax == 1 ? Dy : Dz;
          double tmp[4][4][7];
          gecoef(tmp, lc + 1, ld, Q - C, Q - Dd, kpp.h);
          for (int c = 0; c <= lc + 1; ++c)
            for (int d = 0; d <= ld; ++d)
              for (int t = 0; t < ly.fkT; ++t) FK(ax, c, d, t) = (t & 1) ? -tmp[c][d][t] : tmp[c][d][t];
          for (int c = 0; c <= lc; ++c)
            for (int d = 0; d <= ld; ++d)
              for (int t = 0; t < ly.fkT; ++t) {
                double v = 2.0 * kpp.alpha * ((t & 1) ? -tmp[c + 1][d][t] : tmp[c + 1][d][t]);
                if (c > 0) v -= c * ((t & 1) ? -tmp[c - 1][d][t] : tmp[c - 1][d][t]);
                DC(ax, c, d, t) = v;
              }
        }
        // Boys and R up to L+1
        const double r = rsqrt(bpp.p + kpp.p);
        const double rho = bpp.p * kpp.p * (r * r);
        const double X = bpp.Px - kpp.Px, Y = bpp.Py - kpp.Py, Z = bpp.Pz - kpp.Pz;
        const double tb = rho * (X * X + Y * Y + Z * Z);
        const int L1 = L + 1;
        if (lane <= L1) {
          double pref = 4.0 * kTwoPi25 * bpp.K * kpp.K * (bpp.h * kpp.h) * r;
          for (int k = 0; k < lane; ++k) pref *= -2.0 * rho;
          sRn[lane] = pref * boys_single<double>(tb, lane, prm.boys);
        }
        __syncwarp();
        if (lane == 0) sR[0] = sRn[L1];
        __syncwarp();
        for (int m = L1 - 1; m >= 0; --m) {
          for (int s = L1 - m; s >= 1; --s) {
            const int base_s = s * (s + 1) * (s + 2) / 6;
            for (int k = lane; k < ncart(s); k += 32) {
              int t, u, v;
              wcart(s, k, t, u, v);
              double val;
              if (t > 0) {
                val = X * sR[herm_index(t - 1, u, v)];
                if (t > 1) val += (t - 1) * sR[herm_index(t - 2, u, v)];
              } else if (u > 0) {
                val = Y * sR[herm_index(t, u - 1, v)];
                if (u > 1) val += (u - 1) * sR[herm_index(t, u - 2, v)];
              } else {
                val = Z * sR[herm_index(t, u, v - 1)];
                if (v > 1) val += (v - 1) * sR[herm_index(t, u, v - 2)];
              }
              sR[base_s + k] = val;
            }
            __syncwarp();
          }
          if (lane == 0) sR[0] = sRn[m];
          __syncwarp();
        }
        // stage 1: X[cd][h], h < nherm(lab+1)
        for (int idx = lane; idx < ncd * nh1; idx += 32) {
          const int cd = idx / nh1, h = idx % nh1;
          int t, u, v, cx, cy, cz, dx, dy, dz;
          wherm(h, t, u, v);
          wcart(lc, cd / nd, cx, cy, cz);
          wcart(ld, cd % nd, dx, dy, dz);
          double x = 0.0;
          for (int tp = 0; tp <= cx + dx; ++tp)
            for (int up = 0; up <= cy + dy; ++up) {
              const double fxy = FK(0, cx, dx, tp) * FK(1, cy, dy, up);
              for (int vp = 0; vp <= cz + dz; ++vp) x += fxy * FK(2, cz, dz, vp) * sR[herm_index(t + tp, u + up, v + vp)];
            }
          sX[idx] = x;
        }
        __syncwarp();
        // bra derivatives (A, B)
        for (int e = lane; e < ntot; e += 32) {
          const double w = sG[e];
          if (w == 0.0) continue;
          const int ab = e / ncd, cd = e % ncd;
          int ax, ay, az, bx, by, bz;
          wcart(la, ab / nb, ax, ay, az);
          wcart(lb, ab % nb, bx, by, bz);
          const double* Xc = sX + cd * nh1;
          double sacc[6] = {0, 0, 0, 0, 0, 0};
          for (int t = 0; t <= ax + bx + 1; ++t)
            for (int u = 0; u <= ay + by + 1; ++u)
              for (int v = 0; v <= az + bz + 1; ++v) {
                // exactly one axis may exceed its plain range
                const int over = (t > ax + bx) + (u > ay + by) + (v > az + bz);
                if (over > 1) continue;
                const double xv = Xc[herm_index(t, u, v)];
                const double ex = t <= ax + bx ? EB(0, ax, bx, t) : 0.0;
                const double ey = u <= ay + by ? EB(1, ay, by, u) : 0.0;
                const double ez = v <= az + bz ? EB(2, az, bz, v) : 0.0;
                if (u <= ay + by && v <= az + bz) {
                  sacc[0] += DA(0, ax, bx, t) * ey * ez * xv;
                  sacc[3] += DB(0, ax, bx, t) * ey * ez * xv;
                }
                if (t <= ax + bx && v <= az + bz) {
                  sacc[1] += ex * DA(1, ay, by, u) * ez * xv;
                  sacc[4] += ex * DB(1, ay, by, u) * ez * xv;
                }
                if (t <= ax + bx && u <= ay + by) {
                  sacc[2] += ex * ey * DA(2, az, bz, v) * xv;
                  sacc[5] += ex * ey * DB(2, az, bz, v) * xv;
                }
              }
          for (int k = 0; k < 6; ++k) g[k] += w * sacc[k];
        }
        // ket derivative (C), one axis at a time
        for (int dir = 0; dir < 3; ++dir) {
          __syncwarp();
          for (int idx = lane; idx < ncd * nh0; idx += 32) {
            const int cd = idx / nh0, h = idx % nh0;
            int t, u, v, cx, cy, cz, dx, dy, dz;
            wherm(h, t, u, v);
            wcart(lc, cd / nd, cx, cy, cz);
            wcart(ld, cd % nd, dx, dy, dz);
            const int tx = cx + dx + (dir == 0), ty = cy + dy + (dir == 1), tz = cz + dz + (dir == 2);
            double x = 0.0;
            for (int tp = 0; tp <= tx; ++tp)
              for (int up = 0; up <= ty; ++up)
                for (int vp = 0; vp <= tz; ++vp) {
                  const double fx = dir == 0 ? DC(0, cx, dx, tp) : (tp <= cx + dx ? FK(0, cx, dx, tp) : 0.0);
                  const double fy = dir == 1 ? DC(1, cy, dy, up) : (up <= cy + dy ? FK(1, cy, dy, up) : 0.0);
                  const double fz = dir == 2 ? DC(2, cz, dz, vp) : (vp <= cz + dz ? FK(2, cz, dz, vp) : 0.0);
                  x += fx * fy * fz * sR[herm_index(t + tp, u + up, v + vp)];
                }
            sX[idx] = x;
          }
          __syncwarp();
          for (int e = lane; e < ntot; e += 32) {
            const double w = sG[e];
            if (w == 0.0) continue;
            const int ab = e / ncd, cd = e % ncd;
            int ax, ay, az, bx, by, bz;
            wcart(la, ab / nb, ax, ay, az);
            wcart(lb, ab % nb, bx, by, bz);
            const double* Xc = sX + cd * nh0;
            double sacc = 0.0;
            for (int t = 0; t <= ax + bx; ++t)
              for (int u = 0; u <= ay + by; ++u) {
                const double exy = EB(0, ax, bx, t) * EB(1, ay, by, u);
                for (int v = 0; v <= az + bz; ++v) sacc += exy * EB(2, az, bz, v) * Xc[herm_index(t, u, v)];
              }
            g[6 + dir] += w * sacc;
          }
        }
        __syncwarp();
      }
    }
    // reduce over the warp and scatter to the four atoms
    double sc = 4.0;
    if (bp.diag) sc *= 0.5;
    if (kp.diag) sc *= 0.5;
    if (task.bra == kidx) sc *= 0.5;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      double v = g[k];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      g[k] = v * sc;
    }
    if (lane == 0) {
      double* pf = prm.pair_force;
      for (int k = 0; k < 6; ++k) atomicAdd(pf + 6 * task.bra + k, g[k]);
      for (int k = 0; k < 3; ++k) {
        atomicAdd(pf + 6 * kidx + k, g[6 + k]);
        atomicAdd(pf + 6 * kidx + 3 + k, -(g[k] + g[3 + k] + g[6 + k]));
      }
    }
  }
}

// Fold the per-shell-pair forces into the atoms: one thread per pair.
__global__ void pair_force_reduce_kernel(const ShellPair* pairs, int n_pairs, const int* atom,
                                         const double* pair_force, double* grad) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n_pairs) return;
  const ShellPair sp = pairs[p];
  const int ta = atom[sp.a], tb = atom[sp.b];
  const double* f = pair_force + 6 * (size_t)p;
  for (int k = 0; k < 3; ++k) {
    if (f[k] != 0.0) atomicAdd(grad + 3 * ta + k, f[k]);
    if (f[3 + k] != 0.0) atomicAdd(grad + 3 * tb + k, f[3 + k]);
  }
}

cudaError_t launch_pair_force_reduce(const ShellPair* pairs, int n_pairs, const int* atom, const double* pair_force,
                                     double* grad, cudaStream_t s) {
  if (n_pairs <= 0) return cudaSuccess;
  pair_force_reduce_kernel<<<(n_pairs + 255) / 256, 256, 0, s>>>(pairs, n_pairs, atom, pair_force, grad);
  return cudaGetLastError();
}

cudaError_t launch_warp_grad(int la, int lb, int lc, int ld, const GradParams& p, cudaStream_t s) {
  if (p.n_tasks == 0) return cudaSuccess;
  const GradLayout ly(la, lb, lc, ld);
  const size_t sm = (size_t)kGradWarps * ly.total * sizeof(double);
  static size_t configured = 0;
  if (sm > configured) {
    // the largest class, (dd|dd), needs 4 x 36 KB
    cudaError_t e = cudaFuncSetAttribute(warp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)(kGradWarps * GradLayout(2, 2, 2, 2).total * sizeof(double)));
    if (e != cudaSuccess) return e;
    configured = (size_t)kGradWarps * GradLayout(2, 2, 2, 2).total * sizeof(double);
  }
  const unsigned grid = (unsigned)((p.n_tasks + kGradWarps - 1) / kGradWarps);
  warp_grad_kernel<<<grid, 32 * kGradWarps, sm, s>>>(p, la, lb, lc, ld);
  return cudaGetLastError();
}


}  // namespace jqc
