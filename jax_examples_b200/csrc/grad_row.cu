// Row engine for the ERI-derivative adjoint of the classes with a d-shell
// bra pair (dp or dd) at high L.
//
// One warp evaluates one shell quartet at a time (the tasks of a class, a run
// of kets each); lane r owns the bra Cartesian pair ab = r (and r + 32 for dd
// bras).  Gamma_abcd of the quartet sits in the warp's shared memory.  Per
// primitive quartet, lanes 0..2 build the bra E up to (la+1, lb+1) with the
// derivative coefficients DA = 2 alpha E_{i+1} - i E_{i-1}, DB likewise,
// lanes 3..5 the signed ket E up to lc+1 with DC, lanes 0..L+1 the Boys
// values, and R_tuv up to L+1 is built cooperatively in shared memory
// (warp_hermite_R).  Each
// lane then, for its row ab:
//   Fg[h'] = sum_cd Gamma_abcd F^cd_h'            (ket Hermite h' <= lc+ld)
//   Z[h]   = sum_h' Fg[h'] R_{h+h'}                (h <= la+lb+1)
//   dE/dA_x += sum_h DA^x_ab[h] Z[h], ..., dE/dB_z likewise with DB
//   W[h']  = sum_h E^ab_h R_{h+h'}                 (h' <= lc+ld+1)
//   dE/dC_x += sum_cd Gamma_abcd sum_h' DC^x_cd[h'] W[h'], ...
// so Gamma is contracted with the ket E before R (the bra derivatives) and
// the bra E with R before Gamma (the ket derivative): nothing of size
// nab x ncd is formed per primitive quartet.  Every index is a compile-time
// constant except the lane's own (ax, bx, ...), read from shared memory rows.
// The forces are reduced over the warp and added to the per-shell-pair slots
// like the other gradient kernels; dE/dD = -(dA + dB + dC).
#include "warp_engine.cuh"

namespace jqc {

__host__ __device__ constexpr int gr_herm_order(int h) {
  int s = 0;
  while (nherm(s) <= h) ++s;
  return s;
}
__host__ __device__ constexpr int gr_ht(int h) { return cart_lx(gr_herm_order(h), h - nherm(gr_herm_order(h) - 1)); }
__host__ __device__ constexpr int gr_hu(int h) { return cart_ly(gr_herm_order(h), h - nherm(gr_herm_order(h) - 1)); }
__host__ __device__ constexpr int gr_hv(int h) { return gr_herm_order(h) - gr_ht(h) - gr_hu(h); }

template <int LA, int LB, int LC, int LD>
struct GRowSmem {
  static constexpr int LAB = LA + LB, LCD = LC + LD, L = LAB + LCD;
  static constexpr int NAB = ncart(LA) * ncart(LB), NCD = ncart(LC) * ncart(LD);
  double Eb[3][LA + 2][LB + 2][LAB + 3];  // bra E, i <= la+1, j <= lb+1; zero beyond t = i+j
  double DA[3][LA + 1][LB + 1][LAB + 2];  // derivative on centre A, t <= i+j+1
  double DB[3][LA + 1][LB + 1][LAB + 2];  // derivative on centre B
  double Fk[3][LC + 2][LD + 1][LCD + 2];  // ket E with (-1)^t, c <= lc+1
  double DC[3][LC + 1][LD + 1][LCD + 2];  // derivative on centre C (signed)
  double R[nherm(L + 1)];
  double Rn[L + 2];
  double G[NAB * NCD];                    // Gamma_abcd
};

constexpr int kGRowWarps = 4;

struct F6 {
  double v[6];
};
struct F3 {
  double v[3];
};

// Bra-centre forces of row ab for the current primitive quartet:
// Fg = Gamma_ab. contracted with the ket E, Z = Fg * R, then DA / DB.
template <int LA, int LB, int LC, int LD>
__device__ __noinline__ F6 row_bra(const GRowSmem<LA, LB, LC, LD>* sm, int ab) {
  using S = GRowSmem<LA, LB, LC, LD>;
  constexpr int LAB = S::LAB, LCD = S::LCD, NCD = S::NCD;
  constexpr int NB = ncart(LB), ND = ncart(LD);
  constexpr int NH1 = nherm(LAB + 1), NK0 = nherm(LCD);
  const int ai = ab / NB, bi = ab - (ab / NB) * NB;
  const int ax = cart_lx(LA, ai), ay = cart_ly(LA, ai), az = LA - ax - ay;
  const int bx = cart_lx(LB, bi), by = cart_ly(LB, bi), bz = LB - bx - by;
  const double* Gr = sm->G + ab * NCD;
  double Fg[NK0];
  static_for<NK0>([&](auto h_) { Fg[decltype(h_)::value] = 0.0; });
  static_for<NCD>([&](auto cd_) {
    constexpr int cd = decltype(cd_)::value, ci = cd / ND, di = cd % ND;
    constexpr int cx = cart_lx(LC, ci), cy = cart_ly(LC, ci), cz = cart_lz(LC, ci);
    constexpr int dx = cart_lx(LD, di), dy = cart_ly(LD, di), dz = cart_lz(LD, di);
    const double w = Gr[cd];
    static_for<cx + dx + 1>([&](auto t_) {
      constexpr int t = decltype(t_)::value;
      static_for<cy + dy + 1>([&](auto u_) {
        constexpr int u = decltype(u_)::value;
        const double wxy = w * sm->Fk[0][cx][dx][t] * sm->Fk[1][cy][dy][u];
        static_for<cz + dz + 1>([&](auto v_) {
          constexpr int v = decltype(v_)::value;
          Fg[herm_index(t, u, v)] += wxy * sm->Fk[2][cz][dz][v];
        });
      });
    });
  });
  double ex[LAB + 2], ey[LAB + 2], ez[LAB + 2];
  double dax[LAB + 2], day[LAB + 2], daz[LAB + 2], dbx[LAB + 2], dby[LAB + 2], dbz[LAB + 2];
  static_for<LAB + 2>([&](auto t_) {
    constexpr int t = decltype(t_)::value;
    ex[t] = sm->Eb[0][ax][bx][t];
    ey[t] = sm->Eb[1][ay][by][t];
    ez[t] = sm->Eb[2][az][bz][t];
    dax[t] = sm->DA[0][ax][bx][t];
    day[t] = sm->DA[1][ay][by][t];
    daz[t] = sm->DA[2][az][bz][t];
    dbx[t] = sm->DB[0][ax][bx][t];
    dby[t] = sm->DB[1][ay][by][t];
    dbz[t] = sm->DB[2][az][bz][t];
  });
  // Z[h] = sum_k Fg[k] R_{h+k}: k outer, so the NH1 sums are independent
  double Z[NH1];
  static_for<NH1>([&](auto h_) { Z[decltype(h_)::value] = 0.0; });
  static_for<NK0>([&](auto k_) {
    constexpr int k = decltype(k_)::value;
    const double f = Fg[k];
    static_for<NH1>([&](auto h_) {
      constexpr int h = decltype(h_)::value;
      Z[h] += f * sm->R[herm_index(gr_ht(h) + gr_ht(k), gr_hu(h) + gr_hu(k), gr_hv(h) + gr_hv(k))];
    });
  });
  // The six derivative sums factor through one partial sum per axis:
  // dA_x = sum_t DA^x_t S^x_t with S^x_t = sum_{u,v} E^y_u E^z_v Z_tuv, and
  // likewise for y, z and the B centre.
  double sx[LAB + 2], sy[LAB + 2], sz[LAB + 2];
  static_for<LAB + 2>([&](auto t_) {
    constexpr int t = decltype(t_)::value;
    sx[t] = 0.0;
    sy[t] = 0.0;
    sz[t] = 0.0;
  });
  static_for<NH1>([&](auto h_) {
    constexpr int h = decltype(h_)::value;
    constexpr int t = gr_ht(h), u = gr_hu(h), v = gr_hv(h);
    const double z = Z[h];
    sx[t] += (ey[u] * ez[v]) * z;
    sy[u] += (ex[t] * ez[v]) * z;
    sz[v] += (ex[t] * ey[u]) * z;
  });
  F6 out = {{0, 0, 0, 0, 0, 0}};
  static_for<LAB + 2>([&](auto t_) {
    constexpr int t = decltype(t_)::value;
    out.v[0] += dax[t] * sx[t];
    out.v[1] += day[t] * sy[t];
    out.v[2] += daz[t] * sz[t];
    out.v[3] += dbx[t] * sx[t];
    out.v[4] += dby[t] * sy[t];
    out.v[5] += dbz[t] * sz[t];
  });
  return out;
}

// Ket-centre (C) force of row ab: W = E^ab * R, then Gamma with DC.
template <int LA, int LB, int LC, int LD>
__device__ __noinline__ F3 row_ket(const GRowSmem<LA, LB, LC, LD>* sm, int ab) {
  using S = GRowSmem<LA, LB, LC, LD>;
  constexpr int LAB = S::LAB, LCD = S::LCD, NCD = S::NCD;
  constexpr int NB = ncart(LB), ND = ncart(LD);
  constexpr int NH0 = nherm(LAB), NK1 = nherm(LCD + 1);
  const int ai = ab / NB, bi = ab - (ab / NB) * NB;
  const int ax = cart_lx(LA, ai), ay = cart_ly(LA, ai), az = LA - ax - ay;
  const int bx = cart_lx(LB, bi), by = cart_ly(LB, bi), bz = LB - bx - by;
  const double* Gr = sm->G + ab * NCD;
  double Gab[NH0];
  {
    double ex[LAB + 1], ey[LAB + 1], ez[LAB + 1];
    static_for<LAB + 1>([&](auto t_) {
      constexpr int t = decltype(t_)::value;
      ex[t] = sm->Eb[0][ax][bx][t];
      ey[t] = sm->Eb[1][ay][by][t];
      ez[t] = sm->Eb[2][az][bz][t];
    });
    static_for<NH0>([&](auto h_) {
      constexpr int h = decltype(h_)::value;
      Gab[h] = ex[gr_ht(h)] * ey[gr_hu(h)] * ez[gr_hv(h)];
    });
  }
  // W[k] = sum_h Gab[h] R_{h+k}: h outer, so the NK1 sums are independent
  double W[NK1];
  static_for<NK1>([&](auto k_) { W[decltype(k_)::value] = 0.0; });
  static_for<NH0>([&](auto h_) {
    constexpr int h = decltype(h_)::value;
    const double gh = Gab[h];
    static_for<NK1>([&](auto k_) {
      constexpr int k = decltype(k_)::value;
      W[k] += gh * sm->R[herm_index(gr_ht(h) + gr_ht(k), gr_hu(h) + gr_hu(k), gr_hv(h) + gr_hv(k))];
    });
  });
  F3 out = {{0, 0, 0}};
  static_for<NCD>([&](auto cd_) {
    constexpr int cd = decltype(cd_)::value, ci = cd / ND, di = cd % ND;
    constexpr int cx = cart_lx(LC, ci), cy = cart_ly(LC, ci), cz = cart_lz(LC, ci);
    constexpr int dx = cart_lx(LD, di), dy = cart_ly(LD, di), dz = cart_lz(LD, di);
    constexpr int TX = cx + dx, TY = cy + dy, TZ = cz + dz;
    const double w = Gr[cd];
    // dE/dC_x = sum_t DC^x_t sum_u F^y_u sum_v F^z_v W_tuv (y, z likewise),
    // factored through P_tu = sum_v F^z_v W_tuv and Q_v = sum_{t,u} F^x_t F^y_u W_tuv
    double P[TX + 2][TY + 2];
    static_for<TX + 2>([&](auto t_) {
      constexpr int t = decltype(t_)::value;
      static_for<TY + 2>([&](auto u_) {
        constexpr int u = decltype(u_)::value;
        if constexpr (t <= TX || u <= TY) {
          double acc = 0.0;
          static_for<TZ + 1>([&](auto v_) {
            constexpr int v = decltype(v_)::value;
            acc += sm->Fk[2][cz][dz][v] * W[herm_index(t, u, v)];
          });
          P[t][u] = acc;
        }
      });
    });
    double sx = 0.0, sy = 0.0, sz = 0.0;
    static_for<TX + 2>([&](auto t_) {
      constexpr int t = decltype(t_)::value;
      double a = 0.0;
      static_for<TY + 1>([&](auto u_) {
        constexpr int u = decltype(u_)::value;
        a += sm->Fk[1][cy][dy][u] * P[t][u];
      });
      sx += sm->DC[0][cx][dx][t] * a;
    });
    static_for<TY + 2>([&](auto u_) {
      constexpr int u = decltype(u_)::value;
      double a = 0.0;
      static_for<TX + 1>([&](auto t_) {
        constexpr int t = decltype(t_)::value;
        a += sm->Fk[0][cx][dx][t] * P[t][u];
      });
      sy += sm->DC[1][cy][dy][u] * a;
    });
    static_for<TZ + 2>([&](auto v_) {
      constexpr int v = decltype(v_)::value;
      double q = 0.0;
      static_for<TX + 1>([&](auto t_) {
        constexpr int t = decltype(t_)::value;
        double a = 0.0;
        static_for<TY + 1>([&](auto u_) {
          constexpr int u = decltype(u_)::value;
          a += sm->Fk[1][cy][dy][u] * W[herm_index(t, u, v)];
        });
        q += sm->Fk[0][cx][dx][t] * a;
      });
      sz += sm->DC[2][cz][dz][v] * q;
    });
    out.v[0] += w * sx;
    out.v[1] += w * sy;
    out.v[2] += w * sz;
  });
  return out;
}

// Resident blocks per SM the register allocation aims at: 3 (<= 168
// registers, a few KB of spills) pays for the dp bras and (dd|ps); the other
// dd-bra classes are limited by shared memory anyway and lose to the spills.
__host__ __device__ constexpr int grad_row_min_blocks(int la, int lb, int lc, int ld) {
  return (lb == 1 || (lb == 2 && lc == 1 && ld == 0)) ? 3 : 1;
}

template <int LA, int LB, int LC, int LD>
__global__ void __launch_bounds__(32 * kGRowWarps, grad_row_min_blocks(LA, LB, LC, LD))
    grad_row_kernel(const GradParams prm) {
  using S = GRowSmem<LA, LB, LC, LD>;
  constexpr int LAB = S::LAB, LCD = S::LCD, L = S::L, NAB = S::NAB, NCD = S::NCD;
  constexpr int NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
  constexpr int NH1 = nherm(LAB + 1), NH0 = nherm(LAB), NK0 = nherm(LCD), NK1 = nherm(LCD + 1);
  extern __shared__ __align__(16) unsigned char gr_smraw[];
  S* sm = reinterpret_cast<S*>(gr_smraw) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (warp >= prm.n_tasks) return;
  // entries beyond the valid t of every E array stay zero: clear them once
  for (int i = lane; i < int(sizeof(sm->Eb) / 8); i += 32) (&sm->Eb[0][0][0][0])[i] = 0.0;
  for (int i = lane; i < int(sizeof(sm->DA) / 8); i += 32) (&sm->DA[0][0][0][0])[i] = 0.0;
  for (int i = lane; i < int(sizeof(sm->DB) / 8); i += 32) (&sm->DB[0][0][0][0])[i] = 0.0;
  for (int i = lane; i < int(sizeof(sm->Fk) / 8); i += 32) (&sm->Fk[0][0][0][0])[i] = 0.0;
  for (int i = lane; i < int(sizeof(sm->DC) / 8); i += 32) (&sm->DC[0][0][0][0])[i] = 0.0;
  __syncwarp();
  const Task task = prm.tasks[warp];
  const ShellPair bp = prm.pairs[task.bra];
  const double* ctr = prm.centres;
  const double Ax = ctr[3 * bp.a], Ay = ctr[3 * bp.a + 1], Az = ctr[3 * bp.a + 2];
  const double Bx = ctr[3 * bp.b], By = ctr[3 * bp.b + 1], Bz = ctr[3 * bp.b + 2];
  const int n = prm.n;
  const int a0 = prm.ao[bp.a], b0 = prm.ao[bp.b];
  const int p0 = task.flags & 0xffff, p1 = task.flags >> 16;  // bra primitive-pair range

  for (int kk = 0; kk < task.nket; ++kk) {
    const int kidx = task.ket0 + kk;
    const ShellPair kp = prm.pairs[kidx];
    if (prm.dmax_top != nullptr && float(bp.Q) * float(kp.Q) * gamma_bound_top(prm, *prm.dmax_top) < prm.dens_tau)
      continue;  // warp-uniform
    if (prm.dmax != nullptr && float(bp.Q) * float(kp.Q) * gamma_bound(prm, bp.a, bp.b, kp.a, kp.b) < prm.dens_tau)
      continue;  // warp-uniform
    const double Cx = ctr[3 * kp.a], Cy = ctr[3 * kp.a + 1], Cz = ctr[3 * kp.a + 2];
    const double Dx = ctr[3 * kp.b], Dy = ctr[3 * kp.b + 1], Dz = ctr[3 * kp.b + 2];
    const int c0 = prm.ao[kp.a], d0 = prm.ao[kp.b];
    __syncwarp();
    for (int e = lane; e < NAB * NCD; e += 32) {
      const int ab = e / NCD, cd = e - (e / NCD) * NCD;
      const int ia = a0 + ab / NB, ib = b0 + ab % NB, ic = c0 + cd / ND, id = d0 + cd % ND;
      double dab = 0.0, dcd = 0.0, kx = 0.0;
      for (int s = 0; s < prm.n_dens; ++s) {
        const double* Ds = prm.D + (size_t)s * n * n;
        dab += __ldg(Ds + (size_t)ia * n + ib);
        dcd += __ldg(Ds + (size_t)ic * n + id);
        kx += __ldg(Ds + (size_t)ia * n + ic) * __ldg(Ds + (size_t)ib * n + id) +
              __ldg(Ds + (size_t)ia * n + id) * __ldg(Ds + (size_t)ib * n + ic);
      }
      sm->G[e] = prm.jscale * dab * dcd - 0.5 * prm.kscale * kx;
    }
    double g[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) g[k] = 0.0;

    for (int ip = p0; ip < p1; ++ip) {
      const PrimPair bpp = ld_pp(prm.pp + bp.pp + ip);
      __syncwarp();
      if (lane < 3) {
        const double P = lane == 0 ? bpp.Px : lane == 1 ? bpp.Py : bpp.Pz;
        const double A = lane == 0 ? Ax : lane == 1 ? Ay : Az;
        const double B = lane == 0 ? Bx : lane == 1 ? By : Bz;
        ecoef_compute<double, LA + 1, LB + 1, false>(sm->Eb[lane], P - A, P - B, bpp.h);
        static_for<LA + 1>([&](auto i_) {
          static_for<LB + 1>([&](auto j_) {
            static_for<LAB + 2>([&](auto t_) {
              constexpr int i = decltype(i_)::value, j = decltype(j_)::value, t = decltype(t_)::value;
              double va = 2.0 * bpp.alpha * sm->Eb[lane][i + 1][j][t];
              if constexpr (i > 0) va -= i * sm->Eb[lane][i - 1][j][t];
              double vb = 2.0 * bpp.beta * sm->Eb[lane][i][j + 1][t];
              if constexpr (j > 0) vb -= j * sm->Eb[lane][i][j - 1][t];
              sm->DA[lane][i][j][t] = va;
              sm->DB[lane][i][j][t] = vb;
            });
          });
        });
      }
      for (int iq = 0; iq < kp.npp; ++iq) {
        const PrimPair kpp = ld_pp(prm.pp + kp.pp + iq);
        if (lane >= 3 && lane < 6) {
          const int ax = lane - 3;
          const double Q = ax == 0 ? kpp.Px : ax == 1 ? kpp.Py : kpp.Pz;
          const double C = ax == 0 ? Cx : ax == 1 ? Cy : Cz;
          const double Dd = ax == 0 ? Dx : ax == 1 ? Dy : Dz;
          ecoef_compute<double, LC + 1, LD, true>(sm->Fk[ax], Q - C, Q - Dd, kpp.h);
          static_for<LC + 1>([&](auto c_) {
            static_for<LD + 1>([&](auto d_) {
              static_for<LCD + 2>([&](auto t_) {
                constexpr int c = decltype(c_)::value, d = decltype(d_)::value, t = decltype(t_)::value;
                double v = 2.0 * kpp.alpha * sm->Fk[ax][c + 1][d][t];
                if constexpr (c > 0) v -= c * sm->Fk[ax][c - 1][d][t];
                sm->DC[ax][c][d][t] = v;
              });
            });
          });
        }
        const double r = rsqrt(bpp.p + kpp.p);
        const double rho = bpp.p * kpp.p * (r * r);
        const double X = bpp.Px - kpp.Px, Y = bpp.Py - kpp.Py, Z = bpp.Pz - kpp.Pz;
        const double tb = rho * (X * X + Y * Y + Z * Z);
        if (lane <= L + 1) {
          double pref = 4.0 * kTwoPi25 * bpp.K * kpp.K * (bpp.h * kpp.h) * r;
          for (int k = 0; k < lane; ++k) pref *= -2.0 * rho;
          sm->Rn[lane] = pref * boys_single<double>(tb, lane, prm.boys);
        }
        __syncwarp();
        warp_hermite_R<double, L + 1>(sm->R, sm->Rn, X, Y, Z, lane);
#pragma unroll 1
        for (int ab = lane; ab < NAB; ab += 32) {
          const F6 fb = row_bra<LA, LB, LC, LD>(sm, ab);
          const F3 fc = row_ket<LA, LB, LC, LD>(sm, ab);
#pragma unroll
          for (int k = 0; k < 6; ++k) g[k] += fb.v[k];
#pragma unroll
          for (int k = 0; k < 3; ++k) g[6 + k] += fc.v[k];
        }
        __syncwarp();
      }
    }
    // reduce over the warp and add to the shell-pair force slots
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

template <int LA, int LB, int LC, int LD>
static cudaError_t launch_grad_row_class(const GradParams& p, cudaStream_t s) {
  if (p.n_tasks == 0) return cudaSuccess;
  const size_t sm = kGRowWarps * sizeof(GRowSmem<LA, LB, LC, LD>);
  static bool configured = false;
  if (!configured) {
    cudaError_t e =
        cudaFuncSetAttribute(grad_row_kernel<LA, LB, LC, LD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    configured = true;
  }
  const unsigned grid = (unsigned)((p.n_tasks + kGRowWarps - 1) / kGRowWarps);
  grad_row_kernel<LA, LB, LC, LD><<<grid, 32 * kGRowWarps, sm, s>>>(p);
  return cudaGetLastError();
}

// Gradient classes with a row-engine kernel (bra pair dp or dd).
#define JQC_FOR_GRAD_ROW_CLASSES(X) \
  X(11, 2, 1, 1, 0)                 \
  X(12, 2, 1, 1, 1)                 \
  X(13, 2, 1, 2, 0)                 \
  X(14, 2, 1, 2, 1)                 \
  X(15, 2, 2, 0, 0)                 \
  X(16, 2, 2, 1, 0)                 \
  X(17, 2, 2, 1, 1)                 \
  X(18, 2, 2, 2, 0)                 \
  X(19, 2, 2, 2, 1)                 \
  X(20, 2, 2, 2, 2)

bool has_grad_row_class(int qc) {
  switch (qc) {
#define X(Q, A, B, C, D) case Q:
    JQC_FOR_GRAD_ROW_CLASSES(X)
#undef X
    return true;
    default:
      return false;
  }
}

cudaError_t launch_grad_row(int qc, const GradParams& p, cudaStream_t s) {
  switch (qc) {
#define X(Q, A, B, C, D) \
  case Q:                \
    return launch_grad_row_class<A, B, C, D>(p, s);
    JQC_FOR_GRAD_ROW_CLASSES(X)
#undef X
    default:
      return cudaErrorNotSupported;
  }
}

}  // namespace jqc
