// FP32 instantiations of the fused ERI + J/K kernel (L <= 4 classes).
#include "jk_impl.cuh"

namespace jqc {

cudaError_t launch_jk32_lo(int qc, const JKParams& p, cudaStream_t s) {
  switch (qc) {
#define X(Q, A, B, C, D) \
  case Q:                \
    return launch_jk_class<float, A, B, C, D>(p, s);
    JQC_FOR_REG_CLASSES_LO(X)
#undef X
    default:
      return cudaErrorNotSupported;
  }
}

}  // namespace jqc
