// Fused ERI + J/K digestion kernel (one template per angular class).
//
// Work mapping: one warp takes one Task = one bra shell pair against up to 32
// consecutive ket shell pairs of one (class, contraction) block; lane i owns
// ket pair ket0+i.  blockIdx.y selects the part of the ket Cartesian pairs a
// thread computes (classes with many components are split so the block fits
// in registers).  The contracted integral block never leaves registers: it is
// contracted with D on the spot and added to J and K.
//
// Digestion (fock.py:31-38 restated with 8-fold symmetry): for a canonical
// quartet with scale s = 1/2 per coincidence (a==b shell, c==d shell,
// bra pair == ket pair), every element v = (ab|cd) adds
//   J[a][b] += 2 s v D[c][d],  J[c][d] += 2 s v D[a][b]
//   K[a][d] += s v D[c][b], K[b][d] += s v D[c][a],
//   K[a][c] += s v D[d][b], K[b][c] += s v D[d][a]
// into accumulators A (J) and B (K); afterwards J = A + A^T, K = B + B^T.
// J[a][b] is summed over the lanes of its bra pair with shuffles before one
// atomic per element; everything else goes to FP64 atomics directly.
//
// Packed warps: in the classes whose bra angular sum is at most 2 (the
// ket-outer loop order, every lane reads its own bra primitives) a warp takes
// a group of tasks with at most 32 kets in all, so short ket runs of several
// bra pairs fill one warp instead of leaving lanes idle.
#pragma once

#include "kernels.cuh"

namespace jqc {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <typename T, int LA, int LB, int LC, int LD, int NS>
struct JKBody {
  const JKParams& prm;
  int warp;
  int lane;
  T (*ebra)[LA + 1][LB + 1][LA + LB + 1];  // warp-private shared memory

  template <int PART>
  __device__ __forceinline__ void run() {
    using Cfg = QCfg<LA, LB, LC, LD, NS, PART>;
    if constexpr (Cfg::NCDP > 0) body<PART>();
  }

  template <int PART>
  __device__ __forceinline__ void body() {
    using Cfg = QCfg<LA, LB, LC, LD, NS, PART>;
    using PPT = typename PPType<T>::type;
    constexpr int NA = Cfg::NA, NB = Cfg::NB, ND = Cfg::ND;
    constexpr int NCDP = Cfg::NCDP;

    // Ket-outer classes read their bra per lane, so one warp may hold the
    // kets of several tasks (a packed group, lanes in task order): lane l
    // belongs to the task whose run of kets covers l.  seg = that task's
    // index in the group (-1 past the last ket).
    constexpr bool kPacked = LA + LB <= kKetOuterMaxLab;
    Task task;
    bool in_range;
    int kidx, seg = 0;
    if constexpr (kPacked) {
      const int g0 = prm.groups ? prm.groups[warp] : warp;
      const int nt = prm.groups ? prm.groups[warp + 1] - g0 : 1;
      const int cnt = lane < nt ? prm.tasks[g0 + lane].nket : 0;
      int incl = cnt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
      }
      const int total = __shfl_sync(0xffffffffu, incl, 31);
      const int start = incl - cnt;
      const unsigned starts = __reduce_or_sync(0xffffffffu, (cnt > 0 && start < 32) ? (1u << start) : 0u);
      in_range = lane < total;
      const unsigned upto = starts & (0xffffffffu >> (31 - lane));
      const int ti = (in_range && upto != 0u) ? __popc(upto) - 1 : 0;
      task = prm.tasks[g0 + ti];
      kidx = task.ket0 + (in_range && upto != 0u ? lane - (31 - __clz(upto)) : 0);
      seg = in_range ? ti : -1;
    } else {
      task = prm.tasks[warp];
      in_range = lane < task.nket;
      kidx = task.ket0 + (in_range ? lane : 0);
    }
    const ShellPair bp = prm.pairs[task.bra];
    const ShellPair kp = prm.pairs[kidx];
    bool active = in_range;
    // a compacted packed group may hold tasks of several molecules
    if (kPacked && prm.mol_active != nullptr && active) active = prm.mol_active[prm.shell_mol[bp.a]] != 0;
    if (prm.dmax_top != nullptr && active && float(bp.Q) * float(kp.Q) * (2.f * *prm.dmax_top) < prm.dens_tau)
      active = false;  // below the bound for any density block: no gathers
    if (prm.dmax != nullptr && active) {
      const float* dm = prm.dmax;
      const int ns = prm.n_shell;
      float m = fmaxf(2.f * dm[bp.a * ns + bp.b], 2.f * dm[kp.a * ns + kp.b]);
      m = fmaxf(m, fmaxf(dm[bp.a * ns + kp.a], dm[bp.a * ns + kp.b]));
      m = fmaxf(m, fmaxf(dm[bp.b * ns + kp.a], dm[bp.b * ns + kp.b]));
      if (float(bp.Q) * float(kp.Q) * m < prm.dens_tau) active = false;
    }
    if (__ballot_sync(0xffffffffu, active) == 0u) return;

    const PPT* pp = static_cast<const PPT*>(prm.pp);
    const double* ctr = prm.centres;
    Vec3<T> A{T(ctr[3 * bp.a]), T(ctr[3 * bp.a + 1]), T(ctr[3 * bp.a + 2])};
    Vec3<T> B{T(ctr[3 * bp.b]), T(ctr[3 * bp.b + 1]), T(ctr[3 * bp.b + 2])};
    Vec3<T> C{T(ctr[3 * kp.a]), T(ctr[3 * kp.a + 1]), T(ctr[3 * kp.a + 2])};
    Vec3<T> D{T(ctr[3 * kp.b]), T(ctr[3 * kp.b + 1]), T(ctr[3 * kp.b + 2])};

    T out[Cfg::NAB][Cfg::CDP];
    const int p0 = task.flags & 0xffff, p1 = task.flags >> 16;  // bra primitive-pair range
    quartet_accumulate<T, LA, LB, LC, LD, NS, PART, true>(pp + bp.pp + p0, p1 - p0, A, B, pp + kp.pp,
                                                           active ? kp.npp : 0, C, D, static_cast<const T*>(prm.boys_al),
                                                           ebra, out);

    double s = active ? 1.0 : 0.0;
    if (bp.diag) s *= 0.5;
    if (kp.diag) s *= 0.5;
    if (task.bra == kidx) s *= 0.5;

    // Segmented suffix sums over lanes of one task (packed warps): bit k of
    // vmask says lane + 2^k holds the same task; the first lane of each task
    // ends with its task's total.
    unsigned vmask = 0u;
    bool head = lane == 0;
    if constexpr (kPacked) {
#pragma unroll
      for (int k = 0; k < 5; ++k) {
        const int so = __shfl_down_sync(0xffffffffu, seg, 1 << k);
        if (lane + (1 << k) < 32 && so == seg) vmask |= 1u << k;
      }
      const int sp = __shfl_up_sync(0xffffffffu, seg, 1);
      head = seg >= 0 && (lane == 0 || sp != seg);
    }

    const int n = prm.n;
    const int a0 = prm.ao[bp.a], b0 = prm.ao[bp.b], c0 = prm.ao[kp.a], d0 = prm.ao[kp.b];
    for (int dd = 0; dd < prm.n_dens; ++dd) {
      const double* Dm = prm.D + (size_t)dd * n * n;
      double* Jm = prm.J + (size_t)dd * n * n;
      double* Km = prm.K + (size_t)dd * n * n;
      // J[a][b] (warp-uniform target): reduce over lanes first.
      double dcd[NCDP];
      static_for<NCDP>([&](auto cdi_) {
        constexpr int cdi = decltype(cdi_)::value;
        constexpr int cd = Cfg::CD0 + cdi, c = cd / ND, d = cd % ND;
        dcd[cdi] = active ? __ldg(Dm + (size_t)(c0 + c) * n + d0 + d) : 0.0;
      });
      static_for<NA * NB>([&](auto ab_) {
        constexpr int ab = decltype(ab_)::value;
        double acc = 0.0;
        static_for<NCDP>([&](auto cdi_) {
          constexpr int cdi = decltype(cdi_)::value;
          acc += double(out[ab][cdi]) * dcd[cdi];
        });
        acc *= 2.0 * s;
        if constexpr (kPacked) {
#pragma unroll
          for (int k = 0; k < 5; ++k) {
            const double t = __shfl_down_sync(0xffffffffu, acc, 1 << k);
            if ((vmask >> k) & 1u) acc += t;
          }
        } else {
          acc = warp_sum(acc);
        }
        if (head) atomicAdd(Jm + (size_t)(a0 + ab / NB) * n + b0 + ab % NB, acc);
      });
      if (!active) continue;
      // J[c][d]
      double dab[NA * NB];
      static_for<NA * NB>([&](auto ab_) {
        constexpr int ab = decltype(ab_)::value;
        dab[ab] = __ldg(Dm + (size_t)(a0 + ab / NB) * n + b0 + ab % NB);
      });
      static_for<NCDP>([&](auto cdi_) {
        constexpr int cdi = decltype(cdi_)::value;
        constexpr int cd = Cfg::CD0 + cdi, c = cd / ND, d = cd % ND;
        double acc = 0.0;
        static_for<NA * NB>([&](auto ab_) {
          constexpr int ab = decltype(ab_)::value;
          acc += double(out[ab][cdi]) * dab[ab];
        });
        atomicAdd(Jm + (size_t)(c0 + c) * n + d0 + d, 2.0 * s * acc);
      });
      // K: four blocks, for the (c, d) of this part.  Every D element and
      // every K target is touched once per quartet: K[a][d] sums over b and
      // c in registers before its one atomic (not one atomic per (c, d)
      // component), and each D element is loaded once.  D is symmetric, so
      // its elements are read as D[b][c] rather than D[c][b]: the row is the
      // bra's (the same for the lanes of a task) and the lanes' kets spread
      // over the columns of one row, a few cache lines, not one line a lane.
      constexpr int NC = Cfg::NC, CD0 = Cfg::CD0;
      auto in_part = [](int c, int d) { return c * ND + d >= CD0 && c * ND + d < CD0 + NCDP; };
      auto has_c = [&](int c) {
        bool r = false;
        for (int d = 0; d < ND; ++d) r = r || in_part(c, d);
        return r;
      };
      auto has_d = [&](int d) {
        bool r = false;
        for (int c = 0; c < NC; ++c) r = r || in_part(c, d);
        return r;
      };
      // K[a][d] += sum_{b,c} v D[c][b];  K[a][c] += sum_{b,d} v D[d][b]
      double dbc[NB][NC], dbd[NB][ND];
      static_for<NB>([&](auto b_) {
        constexpr int b = decltype(b_)::value;
        static_for<NC>([&](auto c_) {
          constexpr int c = decltype(c_)::value;
          if constexpr (has_c(c)) dbc[b][c] = __ldg(Dm + (size_t)(b0 + b) * n + c0 + c);
        });
        static_for<ND>([&](auto d_) {
          constexpr int d = decltype(d_)::value;
          if constexpr (has_d(d)) dbd[b][d] = __ldg(Dm + (size_t)(b0 + b) * n + d0 + d);
        });
      });
      static_for<NA>([&](auto a_) {
        constexpr int a = decltype(a_)::value;
        static_for<ND>([&](auto d_) {
          constexpr int d = decltype(d_)::value;
          if constexpr (has_d(d)) {
            double acc = 0.0;
            static_for<NB>([&](auto b_) {
              constexpr int b = decltype(b_)::value;
              static_for<NC>([&](auto c_) {
                constexpr int c = decltype(c_)::value;
                if constexpr (in_part(c, d)) acc += double(out[a * NB + b][c * ND + d - CD0]) * dbc[b][c];
              });
            });
            atomicAdd(Km + (size_t)(a0 + a) * n + d0 + d, s * acc);
          }
        });
        static_for<NC>([&](auto c_) {
          constexpr int c = decltype(c_)::value;
          if constexpr (has_c(c)) {
            double acc = 0.0;
            static_for<NB>([&](auto b_) {
              constexpr int b = decltype(b_)::value;
              static_for<ND>([&](auto d_) {
                constexpr int d = decltype(d_)::value;
                if constexpr (in_part(c, d)) acc += double(out[a * NB + b][c * ND + d - CD0]) * dbd[b][d];
              });
            });
            atomicAdd(Km + (size_t)(a0 + a) * n + c0 + c, s * acc);
          }
        });
      });
      // K[b][d] += sum_{a,c} v D[c][a];  K[b][c] += sum_{a,d} v D[d][a]
      // (the bra's second shell has the fewer functions: its sums stay in
      // registers while the D[a][.] elements stream past)
      double kbd[NB][ND], kbc[NB][NC];
      static_for<NB>([&](auto b_) {
        constexpr int b = decltype(b_)::value;
        static_for<ND>([&](auto d_) { kbd[b][decltype(d_)::value] = 0.0; });
        static_for<NC>([&](auto c_) { kbc[b][decltype(c_)::value] = 0.0; });
      });
      static_for<NA>([&](auto a_) {
        constexpr int a = decltype(a_)::value;
        static_for<NC>([&](auto c_) {
          constexpr int c = decltype(c_)::value;
          if constexpr (has_c(c)) {
            const double x = __ldg(Dm + (size_t)(a0 + a) * n + c0 + c);
            static_for<NB>([&](auto b_) {
              constexpr int b = decltype(b_)::value;
              static_for<ND>([&](auto d_) {
                constexpr int d = decltype(d_)::value;
                if constexpr (in_part(c, d)) kbd[b][d] += double(out[a * NB + b][c * ND + d - CD0]) * x;
              });
            });
          }
        });
        static_for<ND>([&](auto d_) {
          constexpr int d = decltype(d_)::value;
          if constexpr (has_d(d)) {
            const double x = __ldg(Dm + (size_t)(a0 + a) * n + d0 + d);
            static_for<NB>([&](auto b_) {
              constexpr int b = decltype(b_)::value;
              static_for<NC>([&](auto c_) {
                constexpr int c = decltype(c_)::value;
                if constexpr (in_part(c, d)) kbc[b][c] += double(out[a * NB + b][c * ND + d - CD0]) * x;
              });
            });
          }
        });
      });
      static_for<NB>([&](auto b_) {
        constexpr int b = decltype(b_)::value;
        static_for<ND>([&](auto d_) {
          constexpr int d = decltype(d_)::value;
          if constexpr (has_d(d)) atomicAdd(Km + (size_t)(b0 + b) * n + d0 + d, s * kbd[b][d]);
        });
        static_for<NC>([&](auto c_) {
          constexpr int c = decltype(c_)::value;
          if constexpr (has_c(c)) atomicAdd(Km + (size_t)(b0 + b) * n + c0 + c, s * kbc[b][c]);
        });
      });
    }
  }
};

// Warps walk the task list with a grid stride: one task per warp when the
// grid covers the list, several (a persistent grid of resident blocks) when
// the launch caps the grid.
template <typename T, int LA, int LB, int LC, int LD>
__global__ void __launch_bounds__(kMaxJKThreads) jk_kernel(const JKParams prm) {
  constexpr int NS = class_split(LA, LB, LC, LD);
  __shared__ T sE[kMaxJKThreads / 32][3][LA + 1][LB + 1][LA + LB + 1];
  const int stride = int((gridDim.x * blockDim.x) >> 5);
  const int n_work = prm.items ? *prm.n_items : (prm.groups ? prm.n_groups : prm.n_tasks);
  for (int w = int((blockIdx.x * blockDim.x + threadIdx.x) >> 5); w < n_work; w += stride) {
    const int warp = prm.items ? prm.items[w] : w;
    JKBody<T, LA, LB, LC, LD, NS> body{prm, warp, int(threadIdx.x & 31), sE[threadIdx.x >> 5]};
    dispatch_part<NS>(blockIdx.y, body);
    __syncwarp();  // every lane is done with the warp's bra E before the next task writes it
  }
}

template <typename T, int LA, int LB, int LC, int LD>
cudaError_t launch_jk_class(const JKParams& p, cudaStream_t s) {
  constexpr int NS = class_split(LA, LB, LC, LD);
  if (p.n_tasks == 0) return cudaSuccess;
  // packed groups only where the kernel reads its bra per lane
  if (p.groups != nullptr && LA + LB > kKetOuterMaxLab) return cudaErrorInvalidValue;
  const int threads = (p.threads == 64 || p.threads == 256) ? p.threads : 128;
  const int wpb = threads / 32;
  long long blocks = ((p.groups ? p.n_groups : p.n_tasks) + wpb - 1) / wpb;
  if (p.persistent || p.items != nullptr) {  // compacted work: the count is known on the device only
    // resident blocks per SM for this block size, times the SM count
    static int occ[3] = {0, 0, 0};
    static int sms = 0;
    const int slot = threads == 64 ? 0 : (threads == 128 ? 1 : 2);
    if (occ[slot] == 0) {
      int dev = 0, o = 0;
      cudaError_t e = cudaGetDevice(&dev);
      if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, jk_kernel<T, LA, LB, LC, LD>, threads, 0);
      if (e != cudaSuccess) return e;
      occ[slot] = o > 0 ? o : 1;
    }
    const long long cap = (long long)occ[slot] * sms;
    if (blocks > cap) blocks = cap;
  }
  dim3 grid((unsigned)blocks, NS);
  jk_kernel<T, LA, LB, LC, LD><<<grid, threads, 0, s>>>(p);
  return cudaGetLastError();
}

// Quartet classes evaluated by the register kernels (L <= 6); (dd|dp) and
// (dd|dd) go to the warp-cooperative engine.
#define JQC_FOR_REG_CLASSES(X) JQC_FOR_REG_CLASSES_LO(X) JQC_FOR_REG_CLASSES_HI(X)
#define JQC_FOR_REG_CLASSES_LO(X) \
  X(0, 0, 0, 0, 0)             \
  X(1, 1, 0, 0, 0)             \
  X(2, 1, 0, 1, 0)             \
  X(3, 1, 1, 0, 0)             \
  X(4, 1, 1, 1, 0)             \
  X(5, 1, 1, 1, 1)             \
  X(6, 2, 0, 0, 0)             \
  X(7, 2, 0, 1, 0)             \
  X(8, 2, 0, 1, 1)             \
  X(9, 2, 0, 2, 0)
#define JQC_FOR_REG_CLASSES_HI(X) \
  X(10, 2, 1, 0, 0)            \
  X(11, 2, 1, 1, 0)            \
  X(12, 2, 1, 1, 1)            \
  X(13, 2, 1, 2, 0)            \
  X(14, 2, 1, 2, 1)            \
  X(15, 2, 2, 0, 0)            \
  X(16, 2, 2, 1, 0)            \
  X(17, 2, 2, 1, 1)            \
  X(18, 2, 2, 2, 0)

// Expand a body over the 21 quartet classes (bra pair class >= ket pair class).
#define JQC_FOR_QUARTET_CLASSES(X) \
  X(0, 0, 0, 0, 0)                 \
  X(1, 1, 0, 0, 0)                 \
  X(2, 1, 0, 1, 0)                 \
  X(3, 1, 1, 0, 0)                 \
  X(4, 1, 1, 1, 0)                 \
  X(5, 1, 1, 1, 1)                 \
  X(6, 2, 0, 0, 0)                 \
  X(7, 2, 0, 1, 0)                 \
  X(8, 2, 0, 1, 1)                 \
  X(9, 2, 0, 2, 0)                 \
  X(10, 2, 1, 0, 0)                \
  X(11, 2, 1, 1, 0)                \
  X(12, 2, 1, 1, 1)                \
  X(13, 2, 1, 2, 0)                \
  X(14, 2, 1, 2, 1)                \
  X(15, 2, 2, 0, 0)                \
  X(16, 2, 2, 1, 0)                \
  X(17, 2, 2, 1, 1)                \
  X(18, 2, 2, 2, 0)                \
  X(19, 2, 2, 2, 1)                \
  X(20, 2, 2, 2, 2)

}  // namespace jqc
