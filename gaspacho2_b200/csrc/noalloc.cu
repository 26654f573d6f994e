// gpl_kernel_mats_noalloc: the kernel matrices of the sparse GP for callers that must not
// allocate device memory.
//
// Who needs it: host code that enqueues work while a CUDA stream is being captured into a
// graph (a cudaMalloc there breaks or invalidates the capture), real-time or embedded loops
// that forbid any allocation after start-up, and plugins inside a framework that owns all
// device memory and hands buffers to its plugins instead of letting them allocate. Such a
// caller passes every input and output as device memory it already has; the only extra
// memory this path needs, the M x M work matrix that holds Kmm and then its Cholesky factor,
// is a fixed array inside the library (below) instead of a cudaMalloc.
//
// Limits and sharing:
//   - M <= GPL_NOALLOC_MAX_M (256): the array is 256 x 256 doubles = 512 KiB and every GPU
//     that loads the library holds it until the process exits. Larger M is refused with
//     GPL_ERR_LIMIT before any work is enqueued.
//   - All calls on one device share that array, and it keeps the last call's contents. Each
//     call overwrites the M x M block it uses before reading it, so nothing needs clearing,
//     but two calls whose kernels overlap on the GPU (different streams, or host threads
//     racing) corrupt each other's factor: serialise them, e.g. on one stream.
//   - Every call on a stream that is not being captured looks up the array's device address
//     (cudaGetSymbolAddress, with the caller's device current) and remembers it per device;
//     a call made while its stream is being captured uses the remembered address, so make
//     one call on the device before any capture begins (a capture with none yet is refused
//     with GPL_ERR_STATE). Looking the address up again outside capture keeps it right after
//     a cudaDeviceReset or in another context, where the module is loaded anew.
//   - A Kmm that is not positive definite (non-positive pivot) leaves its factor zero-filled,
//     as the reference's choldc does; Kmm^-1 k_n and titsias are then inf/NaN and the call
//     still returns GPL_OK (it only enqueues work and never reads results back).
#include <mutex>

#include "gpl_internal.cuh"

namespace {

constexpr int kMaxM = GPL_NOALLOC_MAX_M;
constexpr int kMaxDevices = 64;

// The scratch: Kmm, then its lower Cholesky factor, column-major M x M with ld M.
static __device__ __align__(256) double g_kmm_work[kMaxM * kMaxM];

std::mutex g_mu;
double* g_work_ptr[kMaxDevices] = {nullptr};

// Device address of g_kmm_work on the current device (host code cannot use the symbol's
// name as a pointer: on the host it only stands in for the device object). Looked up anew
// unless `capturing`, when the address remembered from an earlier call is used.
int work_pointer(bool capturing, double** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return GPL_ERR_CUDA;
  if (dev < 0 || dev >= kMaxDevices) return GPL_ERR_LIMIT;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!capturing) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_kmm_work) != cudaSuccess || p == nullptr) return GPL_ERR_CUDA;
    g_work_ptr[dev] = static_cast<double*>(p);
  }
  if (!g_work_ptr[dev]) return GPL_ERR_STATE;
  *out = g_work_ptr[dev];
  return GPL_OK;
}

}  // namespace

extern "C" int gpl_kernel_mats_noalloc(int N, int M, int Q, const double* X, const double* T, const double* rho,
                                       double* Knm, double* KinvKmn, double* titsias, void* stream) {
  if (N <= 0 || M <= 0 || Q <= 0 || !X || !T || !rho || !Knm || !KinvKmn || !titsias) return GPL_ERR_ARG;
  if (M > kMaxM) return GPL_ERR_LIMIT;
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cap) != cudaSuccess) return GPL_ERR_CUDA;
  double* work = nullptr;
  const int rc = work_pointer(cap != cudaStreamCaptureStatusNone, &work);
  if (rc != GPL_OK) return rc;
  const int e = gpl::launch_kernel_mats_raw(st, N, M, Q, X, T, rho, Knm, KinvKmn, titsias, work);
  return e == 0 ? GPL_OK : GPL_ERR_CUDA;
}
