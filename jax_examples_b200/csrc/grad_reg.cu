// Register-path ERI-derivative adjoint kernels (L <= 3 classes).
#include "grad_impl.cuh"

namespace jqc {

cudaError_t launch_grad_reg(int qc, const GradParams& p, cudaStream_t s) {
  switch (qc) {
#define X(Q, A, B, C, D) \
  case Q:                \
    return launch_grad_class<A, B, C, D>(p, s);
    JQC_FOR_GRAD_REG_CLASSES(X)
#undef X
    default:
      return cudaErrorNotSupported;
  }
}

}  // namespace jqc
