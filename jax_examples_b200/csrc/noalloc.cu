// Allocation-free direct J/K entry point.
//
// Some callers cannot allocate device memory at the moment they need a Fock
// build: a Fock builder called from inside a JAX/XLA program (XLA reserves
// most of the GPU up front and owns all device allocation; a foreign
// allocation can fail or force a device-wide synchronization), or a host
// application that runs the SCF in a fixed-memory real-time loop.  They
// create the context and call jqc_jk once at set-up time (that builds the
// work list), and afterwards call jqc_jk_noalloc, which allocates nothing.
//
// The only scratch of this path, the per-shell-pair density maxima used for
// density screening, lives in a file-scope static __device__ array of
// kNoAllocMaxShells^2 floats (1 MiB); every GPU that loads libjqc.so holds
// it until the process exits.  Inputs (D) and outputs (J, K) stay with the
// caller.
#include <mutex>
#include <string>
#include <vector>

#include "kernels.cuh"

namespace jqc {

int ctx_device(const jqc_ctx* c);
int jk_run_preallocated(jqc_ctx* c, int n_dens, const double* D, double* J, double* K, int precision_mode,
                        double mixed_tau, double dens_tau, float* dmax_scratch, size_t dmax_capacity,
                        cudaStream_t s);

constexpr int kNoAllocMaxShells = 512;
static __device__ __align__(256) float g_noalloc_dmax[kNoAllocMaxShells * kNoAllocMaxShells];

// Device address of g_noalloc_dmax on `device`.  The host-side name of the
// array is only a stand-in; the address must come from
// cudaGetSymbolAddress with the device current.  Looked up once per device.
static int noalloc_scratch(int device, float** out) {
  static std::mutex mu;
  static std::vector<float*> addr;
  std::lock_guard<std::mutex> lock(mu);
  if ((int)addr.size() <= device) addr.resize(device + 1, nullptr);
  if (addr[device] == nullptr) {
    int prev = 0;
    JQC_CUDA_CHECK(cudaGetDevice(&prev));
    JQC_CUDA_CHECK(cudaSetDevice(device));
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_dmax);
    const cudaError_t e2 = cudaSetDevice(prev);
    if (e != cudaSuccess) {
      set_error(std::string("jqc_jk_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      return JQC_ERR_CUDA;
    }
    JQC_CUDA_CHECK(e2);
    addr[device] = static_cast<float*>(p);
  }
  *out = addr[device];
  return JQC_OK;
}

}  // namespace jqc

extern "C" int jqc_jk_noalloc(jqc_ctx* ctx, int n_dens, const double* D, double* J, double* K, int precision_mode,
                              double mixed_tau, double dens_tau, void* stream) {
  using namespace jqc;
  if (ctx == nullptr) {
    set_error("jqc_jk_noalloc: null context");
    return JQC_ERR_INVALID;
  }
  float* scratch = nullptr;
  const int rc = noalloc_scratch(ctx_device(ctx), &scratch);
  if (rc) return rc;
  return jk_run_preallocated(ctx, n_dens, D, J, K, precision_mode, mixed_tau, dens_tau, scratch,
                             (size_t)kNoAllocMaxShells * kNoAllocMaxShells, static_cast<cudaStream_t>(stream));
}
