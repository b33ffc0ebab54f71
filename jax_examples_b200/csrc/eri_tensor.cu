// Dense ERI tensor kernels (register classes).
#include "jk_impl.cuh"

namespace jqc {

// ------------------------------------------------------------- dense tensor
// eri.py:69-138: every canonical shell quartet writes its Cartesian block to
// the 8 symmetry-equivalent positions of the (n,n,n,n) tensor.
template <int LA, int LB, int LC, int LD, int NS>
struct TensorBody {
  const TensorParams& prm;
  int warp, lane;
  double (*ebra)[LA + 1][LB + 1][LA + LB + 1];

  template <int PART>
  __device__ __forceinline__ void run() {
    using Cfg = QCfg<LA, LB, LC, LD, NS, PART>;
    if constexpr (Cfg::NCDP > 0) body<PART>();
  }

  template <int PART>
  __device__ __forceinline__ void body() {
    using Cfg = QCfg<LA, LB, LC, LD, NS, PART>;
    constexpr int NA = Cfg::NA, NB = Cfg::NB, ND = Cfg::ND;
    const Task task = prm.tasks[warp];
    const bool active = lane < task.nket;
    const ShellPair bp = prm.pairs[task.bra];
    const ShellPair kp = prm.pairs[task.ket0 + (active ? lane : 0)];
    const double* ctr = prm.centres;
    Vec3<double> A{ctr[3 * bp.a], ctr[3 * bp.a + 1], ctr[3 * bp.a + 2]};
    Vec3<double> B{ctr[3 * bp.b], ctr[3 * bp.b + 1], ctr[3 * bp.b + 2]};
    Vec3<double> C{ctr[3 * kp.a], ctr[3 * kp.a + 1], ctr[3 * kp.a + 2]};
    Vec3<double> D{ctr[3 * kp.b], ctr[3 * kp.b + 1], ctr[3 * kp.b + 2]};
    double out[Cfg::NAB][Cfg::CDP];
    quartet_accumulate<double, LA, LB, LC, LD, NS, PART, true>(prm.pp + bp.pp, bp.npp, A, B, prm.pp + kp.pp,
                                                                active ? kp.npp : 0, C, D, prm.boys_al, ebra, out);
    if (!active) return;
    const long long n = prm.n;
    const long long a0 = prm.ao[bp.a], b0 = prm.ao[bp.b], c0 = prm.ao[kp.a], d0 = prm.ao[kp.b];
    double* e = prm.eri;
    static_for<NA * NB * Cfg::NCDP>([&](auto x_) {
          constexpr int x = decltype(x_)::value;
          constexpr int ab = x / Cfg::NCDP, cdi = x % Cfg::NCDP, a = ab / NB, b = ab % NB;
          constexpr int cd = Cfg::CD0 + cdi, c = cd / ND, d = cd % ND;
          const double v = out[ab][cdi];
          const long long i = a0 + a, j = b0 + b, k = c0 + c, l = d0 + d;
          e[((i * n + j) * n + k) * n + l] = v;
          e[((j * n + i) * n + k) * n + l] = v;
          e[((i * n + j) * n + l) * n + k] = v;
          e[((j * n + i) * n + l) * n + k] = v;
          e[((k * n + l) * n + i) * n + j] = v;
          e[((l * n + k) * n + i) * n + j] = v;
          e[((k * n + l) * n + j) * n + i] = v;
          e[((l * n + k) * n + j) * n + i] = v;
        });
  }
};

template <int LA, int LB, int LC, int LD>
__global__ void __launch_bounds__(128) tensor_kernel(const TensorParams prm) {
  constexpr int NS = class_split(LA, LB, LC, LD);
  __shared__ double sE[4][3][LA + 1][LB + 1][LA + LB + 1];
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (warp >= prm.n_tasks) return;
  TensorBody<LA, LB, LC, LD, NS> body{prm, warp, int(threadIdx.x & 31), sE[threadIdx.x >> 5]};
  dispatch_part<NS>(blockIdx.y, body);
}

cudaError_t launch_eri_tensor(int qc, const TensorParams& p, cudaStream_t s) {
  if (p.n_tasks == 0) return cudaSuccess;
  if (!is_reg_class(qc)) {
    const int pb = qc_bra(qc), pk = qc_ket(qc);
    return launch_warp_tensor(pc_la(pb), pc_lb(pb), pc_la(pk), pc_lb(pk), p, s);
  }
  switch (qc) {
#define X(Q, A, B, C, D)                                                                     \
  case Q: {                                                                                  \
    dim3 grid((p.n_tasks + 3) / 4, class_split(A, B, C, D));                                 \
    tensor_kernel<A, B, C, D><<<grid, 128, 0, s>>>(p);                                       \
    return cudaGetLastError();                                                               \
  }
    JQC_FOR_REG_CLASSES(X)
#undef X
    default:
      return cudaErrorInvalidValue;
  }
}

}  // namespace jqc
