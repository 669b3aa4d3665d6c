// noalloc.cu -- calaman_expm_noalloc_d: exp(A) for double matrices up to
// kNoAllocMaxN x kNoAllocMaxN without any device allocation by the caller.
//
// Some callers cannot call cudaMalloc: code hosted by a framework that owns
// every device allocation and hands out none, loops that must not allocate
// once they are running, and small FFI or plugin callers with no device
// allocator at hand. The call also creates no stream or event: its LU runs
// every panel on the caller's stream. This entry point serves them by running the ordinary
// calaman_expm_d on a workspace that lives in a file-scope device array of
// this library, so the caller passes only the input, the output and d_info.
//
// The array is kNoAllocScratchBytes (4 MiB) and every GPU that loads the
// library holds it until the process exits. Its device address is looked up
// once per device, on the first call made with that device current; make that
// first call before any stream capture. The address is kept for the life of
// the process: a cudaDeviceReset after the first call on a device (which
// reloads the module into a new context, where the array may sit elsewhere)
// is not supported. Like calaman_expm_d, every call synchronises its stream
// once, to read the 1-norm back for the (m, s) plan; a caller that already
// knows the plan and must not synchronise uses calaman_pade_d and the
// squarings itself. Every call shares the one array, so
// calls that overlap on the GPU (other streams, other host threads) race on
// it; serialise them. Nothing in the array needs to start at zero: each call
// initialises everything it reads, and the array keeps the last call's data.
#include <mutex>

#include "kernels.cuh"

namespace {

constexpr int kNoAllocMaxN = 256;
constexpr std::size_t kNoAllocScratchBytes = std::size_t(4) << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_expm_scratch[kNoAllocScratchBytes];

std::mutex g_mu;
void *g_scratch_ptr[kMaxDevices] = {};

// The device address of g_expm_scratch on the current device (looked up once).
calamanStatus_t scratch_for_current_device(void **out) {
  int dev = 0;
  CLM_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return clm::blas_status(CALAMAN_STATUS_NOT_SUPPORTED);
  std::lock_guard<std::mutex> lock(g_mu);
  if (g_scratch_ptr[dev] == nullptr) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_expm_scratch);
    if (e != cudaSuccess) return clm::runtime_status(e);
    if (p == nullptr) return clm::blas_status(CALAMAN_STATUS_INTERNAL_ERROR);
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return clm::ok_status();
}

}  // namespace

extern "C" calamanStatus_t calaman_expm_noalloc_d(calamanBlasHandle_t blas, calamanStream_t stream,
                                                  int n, const double *d_A, int lda,
                                                  double *d_expA, int lde, int *d_info,
                                                  calamanExpmPlan_t *plan) {
  if (n < 1 || lda < n || lde < n || d_A == nullptr || d_expA == nullptr || d_info == nullptr)
    return clm::blas_status(CALAMAN_STATUS_INVALID_VALUE);
  if (n > kNoAllocMaxN) return clm::blas_status(CALAMAN_STATUS_NOT_SUPPORTED);
  size_t need = 0;
  CLM_TRY(calaman_expm_bufferSize_d(blas, n, &need));
  if (need > kNoAllocScratchBytes) return clm::blas_status(CALAMAN_STATUS_NOT_SUPPORTED);
  void *scratch = nullptr;
  CLM_TRY(scratch_for_current_device(&scratch));
  // no look-ahead stream either: this path creates no CUDA resources
  clm::NoLookAheadScope serial;
  return calaman_expm_d(blas, blas, stream, n, d_A, lda, d_expA, lde, scratch, kNoAllocScratchBytes,
                        d_info, plan);
}
