// Register-path ERI-derivative adjoint kernel (classes with L <= 4).
//
// Same mathematics as warp_grad_kernel (grad.cu), with the class unrolled at
// compile time and the work mapping of the J/K kernels: one warp per bra
// pair and up to 32 ket pairs, one lane per shell quartet, blockIdx.y
// selecting the part of the ket Cartesian pairs a thread handles.  The bra
// E coefficients up to (la+1, lb+1) and the derivative coefficients DA, DB
// live in warp-shared memory (the bra is warp-uniform); Gamma for the
// thread's part, the ket E/DC coefficients, R up to L+1 and the nine force
// components live in registers.  Forces on the bra centres are reduced over
// the warp before the atomics; the ket centres' go straight to atomics.
#pragma once

#include "jk_impl.cuh"

namespace jqc {

__host__ __device__ constexpr int grad_split(int la, int lb, int lc, int ld) {
  int nab = ncart(la) * ncart(lb), ncd = ncart(lc) * ncart(ld);
  int ns = 1;
  while (ns < 16 && nab * ((ncd + ns - 1) / ns) > 9 && ns < ncd) ns *= 2;
  return ns;
}

template <int LA, int LB>
struct GradBraSmem {
  double E[3][LA + 2][LB + 2][LA + LB + 3];
  double DA[3][LA + 1][LB + 1][LA + LB + 2];
  double DB[3][LA + 1][LB + 1][LA + LB + 2];
};

// Decode compile-time Hermite index h into (t,u,v).
template <int H>
struct HermDecode {
  static constexpr int s = (H >= 35) ? 5 : (H >= 20) ? 4 : (H >= 10) ? 3 : (H >= 4) ? 2 : (H >= 1) ? 1 : 0;
  static constexpr int k = H - s * (s + 1) * (s + 2) / 6;
  static constexpr int t = cart_lx(s, k), u = cart_ly(s, k), v = s - t - u;
};

template <int LA, int LB, int LC, int LD, int NS>
struct GradBody {
  const GradParams& prm;
  int warp, lane;
  GradBraSmem<LA, LB>* sb;

  // SIDE 0: all forces; 1: bra centres (A, B) only; 2: ket centre C only.
  template <int PART, int SIDE = 0>
  __device__ __forceinline__ void run() {
    using Cfg = QCfg<LA, LB, LC, LD, NS, PART>;
    if constexpr (Cfg::NCDP > 0) body<PART, SIDE>();
  }

  template <int PART, int SIDE>
  __device__ __forceinline__ void body() {
    constexpr bool kBra = SIDE != 2, kKet = SIDE != 1;
    using Cfg = QCfg<LA, LB, LC, LD, NS, PART>;
    constexpr int NA = Cfg::NA, NB = Cfg::NB, ND = Cfg::ND;
    constexpr int NCDP = Cfg::NCDP;
    constexpr int L = Cfg::L, LAB = Cfg::LAB;
    constexpr int NH1 = nherm(LAB + 1), NH0 = nherm(LAB);

    const Task task = prm.tasks[warp];
    const ShellPair bp = prm.pairs[task.bra];
    const bool in_range = lane < task.nket;
    const int kidx = task.ket0 + (in_range ? lane : 0);
    const ShellPair kp = prm.pairs[kidx];
    bool active = in_range;
    if (prm.dmax_top != nullptr && active &&
        float(bp.Q) * float(kp.Q) * gamma_bound_top(prm, *prm.dmax_top) < prm.dens_tau)
      active = false;  // below the bound for any density block: no gathers
    if (prm.dmax != nullptr && active &&
        float(bp.Q) * float(kp.Q) * gamma_bound(prm, bp.a, bp.b, kp.a, kp.b) < prm.dens_tau)
      active = false;
    if (__ballot_sync(0xffffffffu, active) == 0u) return;
    const double* ctr = prm.centres;
    const Vec3<double> A{ctr[3 * bp.a], ctr[3 * bp.a + 1], ctr[3 * bp.a + 2]};
    const Vec3<double> B{ctr[3 * bp.b], ctr[3 * bp.b + 1], ctr[3 * bp.b + 2]};
    const Vec3<double> C{ctr[3 * kp.a], ctr[3 * kp.a + 1], ctr[3 * kp.a + 2]};
    const Vec3<double> Dc{ctr[3 * kp.b], ctr[3 * kp.b + 1], ctr[3 * kp.b + 2]};
    const int n = prm.n;
    const int a0 = prm.ao[bp.a], b0 = prm.ao[bp.b], c0 = prm.ao[kp.a], d0 = prm.ao[kp.b];

    // Gamma for this thread's part
    double G[Cfg::NAB][Cfg::CDP];
    static_for<Cfg::NAB * NCDP>([&](auto x_) {
      constexpr int x = decltype(x_)::value;
      constexpr int ab = x / NCDP, cdi = x % NCDP, cd = Cfg::CD0 + cdi;
      const int ia = a0 + ab / NB, ib = b0 + ab % NB, ic = c0 + cd / ND, id = d0 + cd % ND;
      double dab = 0.0, dcd = 0.0, kx = 0.0;
      if (active) {
        for (int s = 0; s < prm.n_dens; ++s) {
          const double* Ds = prm.D + (size_t)s * n * n;
          dab += __ldg(Ds + (size_t)ia * n + ib);
          dcd += __ldg(Ds + (size_t)ic * n + id);
          kx += __ldg(Ds + (size_t)ia * n + ic) * __ldg(Ds + (size_t)ib * n + id) +
                __ldg(Ds + (size_t)ia * n + id) * __ldg(Ds + (size_t)ib * n + ic);
        }
      }
      G[ab][cdi] = prm.jscale * dab * dcd - 0.5 * prm.kscale * kx;
    });
    double g[9];
    static_for<9>([&](auto k) { g[decltype(k)::value] = 0.0; });
    const int nket = active ? kp.npp : 0;

    const int p0 = task.flags & 0xffff, p1 = task.flags >> 16;  // bra primitive-pair range
    for (int ip = p0; ip < p1; ++ip) {
      const PrimPair bpp = ld_pp(prm.pp + bp.pp + ip);
      __syncwarp();
      if (lane < 3) {
        const double P = lane == 0 ? bpp.Px : lane == 1 ? bpp.Py : bpp.Pz;
        const double a = lane == 0 ? A.x : lane == 1 ? A.y : A.z;
        const double b = lane == 0 ? B.x : lane == 1 ? B.y : B.z;
        ecoef_compute<double, LA + 1, LB + 1, false>(sb->E[lane], P - a, P - b, bpp.h);
        static_for<LA + 1>([&](auto i_) {
          static_for<LB + 1>([&](auto j_) {
            static_for<LA + LB + 2>([&](auto t_) {
              constexpr int i = decltype(i_)::value, j = decltype(j_)::value, t = decltype(t_)::value;
              double va = 2.0 * bpp.alpha * (t <= i + 1 + j ? sb->E[lane][i + 1][j][t] : 0.0);
              if constexpr (i > 0 && t <= i - 1 + j) va -= i * sb->E[lane][i - 1][j][t];
              double vb = 2.0 * bpp.beta * (t <= i + j + 1 ? sb->E[lane][i][j + 1][t] : 0.0);
              if constexpr (j > 0 && t <= i + j - 1) vb -= j * sb->E[lane][i][j - 1][t];
              sb->DA[lane][i][j][t] = va;
              sb->DB[lane][i][j][t] = vb;
            });
          });
        });
      }
      __syncwarp();
      for (int iq = 0; iq < nket; ++iq) {
        const PrimPair kpp = ld_pp(prm.pp + kp.pp + iq);
        double F[3][LC + 2][LD + 1][LC + LD + 2];
        ecoef_compute<double, LC + 1, LD, true>(F[0], kpp.Px - C.x, kpp.Px - Dc.x, kpp.h);
        ecoef_compute<double, LC + 1, LD, true>(F[1], kpp.Py - C.y, kpp.Py - Dc.y, kpp.h);
        ecoef_compute<double, LC + 1, LD, true>(F[2], kpp.Pz - C.z, kpp.Pz - Dc.z, kpp.h);
        double R[nherm(L + 1)];
        prim_quartet_R<double, L + 1>(bpp, kpp, prm.boys_al, R);
        const double two_g = 2.0 * kpp.alpha;

        static_for<NCDP>([&](auto cdi_) {
          constexpr int cdi = decltype(cdi_)::value;
          constexpr int cd = Cfg::CD0 + cdi, c = cd / ND, d = cd % ND;
          constexpr int cx = cart_lx(LC, c), cy = cart_ly(LC, c), cz = cart_lz(LC, c);
          constexpr int dx = cart_lx(LD, d), dy = cart_ly(LD, d), dz = cart_lz(LD, d);
          if constexpr (kBra) {
          // stage 1 with one extra bra Hermite order
          double X[NH1];
          static_for<NH1>([&](auto h) { X[decltype(h)::value] = 0.0; });
          static_for<cx + dx + 1>([&](auto tp_) {
            constexpr int tp = decltype(tp_)::value;
            static_for<cy + dy + 1>([&](auto up_) {
              constexpr int up = decltype(up_)::value;
              const double fxy = F[0][cx][dx][tp] * F[1][cy][dy][up];
              static_for<cz + dz + 1>([&](auto vp_) {
                constexpr int vp = decltype(vp_)::value;
                const double f = fxy * F[2][cz][dz][vp];
                static_for<NH1>([&](auto h_) {
                  constexpr int h = decltype(h_)::value;
                  using Hd = HermDecode<h>;
                  X[h] += f * R[herm_index(Hd::t + tp, Hd::u + up, Hd::v + vp)];
                });
              });
            });
          });
          // bra derivatives
          static_for<NA * NB>([&](auto ab_) {
            constexpr int ab = decltype(ab_)::value, ia = ab / NB, ib = ab % NB;
            constexpr int ax = cart_lx(LA, ia), ay = cart_ly(LA, ia), az = cart_lz(LA, ia);
            constexpr int bx = cart_lx(LB, ib), by = cart_ly(LB, ib), bz = cart_lz(LB, ib);
            double s0 = 0, s1 = 0, s2 = 0, s3 = 0, s4 = 0, s5 = 0;
            // x-derivative terms: t up to ax+bx+1
            static_for<ax + bx + 2>([&](auto t_) {
              constexpr int t = decltype(t_)::value;
              static_for<ay + by + 1>([&](auto u_) {
                constexpr int u = decltype(u_)::value;
                static_for<az + bz + 1>([&](auto v_) {
                  constexpr int v = decltype(v_)::value;
                  const double eyz = sb->E[1][ay][by][u] * sb->E[2][az][bz][v] * X[herm_index(t, u, v)];
                  s0 += sb->DA[0][ax][bx][t] * eyz;
                  s3 += sb->DB[0][ax][bx][t] * eyz;
                });
              });
            });
            static_for<ax + bx + 1>([&](auto t_) {
              constexpr int t = decltype(t_)::value;
              static_for<ay + by + 2>([&](auto u_) {
                constexpr int u = decltype(u_)::value;
                static_for<az + bz + 1>([&](auto v_) {
                  constexpr int v = decltype(v_)::value;
                  const double exz = sb->E[0][ax][bx][t] * sb->E[2][az][bz][v] * X[herm_index(t, u, v)];
                  s1 += sb->DA[1][ay][by][u] * exz;
                  s4 += sb->DB[1][ay][by][u] * exz;
                });
              });
            });
            static_for<ax + bx + 1>([&](auto t_) {
              constexpr int t = decltype(t_)::value;
              static_for<ay + by + 1>([&](auto u_) {
                constexpr int u = decltype(u_)::value;
                static_for<az + bz + 2>([&](auto v_) {
                  constexpr int v = decltype(v_)::value;
                  const double exy = sb->E[0][ax][bx][t] * sb->E[1][ay][by][u] * X[herm_index(t, u, v)];
                  s2 += sb->DA[2][az][bz][v] * exy;
                  s5 += sb->DB[2][az][bz][v] * exy;
                });
              });
            });
            const double w = G[ab][cdi];
            g[0] += w * s0;
            g[1] += w * s1;
            g[2] += w * s2;
            g[3] += w * s3;
            g[4] += w * s4;
            g[5] += w * s5;
          });
          }
          // ket (centre C) derivative, one axis at a time
          if constexpr (kKet) static_for<3>([&](auto dir_) {
            constexpr int dir = decltype(dir_)::value;
            constexpr int ex = cx + dx + (dir == 0), ey = cy + dy + (dir == 1), ez = cz + dz + (dir == 2);
            double Xp[NH0];
            static_for<NH0>([&](auto h) { Xp[decltype(h)::value] = 0.0; });
            static_for<ex + 1>([&](auto tp_) {
              constexpr int tp = decltype(tp_)::value;
              static_for<ey + 1>([&](auto up_) {
                constexpr int up = decltype(up_)::value;
                static_for<ez + 1>([&](auto vp_) {
                  constexpr int vp = decltype(vp_)::value;
                  // derivative factor on axis `dir`, plain (signed) E elsewhere
                  double fx = 0.0, fy = 0.0, fz = 0.0;
                  if constexpr (dir == 0) {
                    if constexpr (tp <= cx + 1 + dx) fx = two_g * F[0][cx + 1][dx][tp];
                    if constexpr (cx > 0 && tp <= cx - 1 + dx) fx -= cx * F[0][cx - 1][dx][tp];
                  } else if constexpr (tp <= cx + dx) {
                    fx = F[0][cx][dx][tp];
                  }
                  if constexpr (dir == 1) {
                    if constexpr (up <= cy + 1 + dy) fy = two_g * F[1][cy + 1][dy][up];
                    if constexpr (cy > 0 && up <= cy - 1 + dy) fy -= cy * F[1][cy - 1][dy][up];
                  } else if constexpr (up <= cy + dy) {
                    fy = F[1][cy][dy][up];
                  }
                  if constexpr (dir == 2) {
                    if constexpr (vp <= cz + 1 + dz) fz = two_g * F[2][cz + 1][dz][vp];
                    if constexpr (cz > 0 && vp <= cz - 1 + dz) fz -= cz * F[2][cz - 1][dz][vp];
                  } else if constexpr (vp <= cz + dz) {
                    fz = F[2][cz][dz][vp];
                  }
                  const double f = fx * fy * fz;
                  static_for<NH0>([&](auto h_) {
                    constexpr int h = decltype(h_)::value;
                    using Hd = HermDecode<h>;
                    Xp[h] += f * R[herm_index(Hd::t + tp, Hd::u + up, Hd::v + vp)];
                  });
                });
              });
            });
            static_for<NA * NB>([&](auto ab_) {
              constexpr int ab = decltype(ab_)::value, ia = ab / NB, ib = ab % NB;
              constexpr int ax = cart_lx(LA, ia), ay = cart_ly(LA, ia), az = cart_lz(LA, ia);
              constexpr int bx = cart_lx(LB, ib), by = cart_ly(LB, ib), bz = cart_lz(LB, ib);
              double s = 0.0;
              static_for<ax + bx + 1>([&](auto t_) {
                constexpr int t = decltype(t_)::value;
                static_for<ay + by + 1>([&](auto u_) {
                  constexpr int u = decltype(u_)::value;
                  const double exy = sb->E[0][ax][bx][t] * sb->E[1][ay][by][u];
                  static_for<az + bz + 1>([&](auto v_) {
                    constexpr int v = decltype(v_)::value;
                    s += exy * sb->E[2][az][bz][v] * Xp[herm_index(t, u, v)];
                  });
                });
              });
              g[6 + dir] += G[ab][cdi] * s;
            });
          });
        });
      }
    }
    // scatter: 4 s per canonical quartet; bra centres reduced over the warp
    double sc = active ? 4.0 : 0.0;
    if (bp.diag) sc *= 0.5;
    if (kp.diag) sc *= 0.5;
    if (task.bra == kidx) sc *= 0.5;
    static_for<9>([&](auto k) { g[decltype(k)::value] *= sc; });
    double* pf = prm.pair_force;
    if constexpr (kBra) {
      static_for<6>([&](auto k_) {
        constexpr int k = decltype(k_)::value;
        const double v = warp_sum(g[k]);
        if (lane == 0) atomicAdd(pf + 6 * task.bra + k, v);
      });
    }
    // centre D by translational invariance: each side adds minus its own part
    if (active) {
      static_for<3>([&](auto k_) {
        constexpr int k = decltype(k_)::value;
        if constexpr (kKet) atomicAdd(pf + 6 * kidx + k, g[6 + k]);
        atomicAdd(pf + 6 * kidx + 3 + k, -((kBra ? g[k] + g[3 + k] : 0.0) + (kKet ? g[6 + k] : 0.0)));
      });
    }
  }
};

// Runs one side of GradBody for the part dispatch_part selects.
template <typename Body, int SIDE>
struct GradSide {
  Body& b;
  template <int PART>
  __device__ __forceinline__ void run() {
    b.template run<PART, SIDE>();
  }
};

// SIDES = 1: one block part per ket Cartesian part computes every force.
// SIDES = 2: the bra-centre and the ket-centre forces run in separate block
// parts (blockIdx.y = 2 * part + side), each with its own R and Boys values,
// so a thread holds only the stage-1 sums of one side (the L = 3, 4 classes
// otherwise spill kilobytes per thread).
template <int LA, int LB, int LC, int LD, int SIDES>
__global__ void __launch_bounds__(128) grad_kernel(const GradParams prm) {
  constexpr int NS = grad_split(LA, LB, LC, LD);
  __shared__ GradBraSmem<LA, LB> sB[4];
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (warp >= prm.n_tasks) return;
  using Body = GradBody<LA, LB, LC, LD, NS>;
  Body body{prm, warp, int(threadIdx.x & 31), &sB[threadIdx.x >> 5]};
  if constexpr (SIDES == 1) {
    dispatch_part<NS>(blockIdx.y, body);
  } else if (blockIdx.y & 1) {
    GradSide<Body, 2> side{body};
    dispatch_part<NS>(blockIdx.y >> 1, side);
  } else {
    GradSide<Body, 1> side{body};
    dispatch_part<NS>(blockIdx.y >> 1, side);
  }
}

template <int LA, int LB, int LC, int LD>
cudaError_t launch_grad_class(const GradParams& p, cudaStream_t s) {
  constexpr int NS = grad_split(LA, LB, LC, LD);
  if (p.n_tasks == 0) return cudaSuccess;
  if (p.sides == 2) {
    dim3 grid((p.n_tasks + 3) / 4, 2 * NS);
    grad_kernel<LA, LB, LC, LD, 2><<<grid, 128, 0, s>>>(p);
  } else {
    dim3 grid((p.n_tasks + 3) / 4, NS);
    grad_kernel<LA, LB, LC, LD, 1><<<grid, 128, 0, s>>>(p);
  }
  return cudaGetLastError();
}

// Classes whose gradient runs in the register kernels.
#define JQC_FOR_GRAD_REG_CLASSES(X) \
  X(0, 0, 0, 0, 0)                  \
  X(1, 1, 0, 0, 0)                  \
  X(2, 1, 0, 1, 0)                  \
  X(3, 1, 1, 0, 0)                  \
  X(4, 1, 1, 1, 0)                  \
  X(6, 2, 0, 0, 0)                  \
  X(7, 2, 0, 1, 0)                  \
  X(10, 2, 1, 0, 0)                 \
  X(5, 1, 1, 1, 1)                  \
  X(8, 2, 0, 1, 1)                  \
  X(9, 2, 0, 2, 0)                  \
  X(11, 2, 1, 1, 0)                 \
  X(15, 2, 2, 0, 0)


}  // namespace jqc
