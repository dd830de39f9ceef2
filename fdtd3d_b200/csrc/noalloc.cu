// noalloc.cu - compensated sum-of-squares reduction that allocates nothing.
//
// Some callers cannot allocate device memory once their run has started:
// an embedding application whose caching allocator already owns the
// device's memory budget, or a real-time step loop where cudaMalloc can
// stall and cudaFree synchronises the whole device.  fdtd_reduce_sq_noalloc
// serves them: the caller passes the input and the output buffers, and the
// per-block partial sums live in a fixed file-scope device array instead of
// memory allocated per call or per context.
//
// The array is kNoAllocMaxBlocks pairs of doubles (16 KiB plus a small
// tail).  Every GPU that loads the library holds it until the process
// exits.  All calls share it, so calls that overlap on the GPU (different
// streams, or different host threads on one device) race on it and must be
// ordered by the caller.  Each call rewrites every partial it reads before
// reading it, so nothing has to be cleared between calls.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/fdtd_b200.h"
#include "kernels.h"

namespace fdtdb {

namespace {

constexpr int kNoAllocMaxBlocks = 1024;

// (sum, compensation) per block; never addressed from host code directly:
// on the host the name is only a stand-in, so its device address is looked
// up per device at set-up.
__device__ __align__ (256) double g_noalloc_partials[2 * kNoAllocMaxBlocks];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
double *g_partials_addr[kMaxDevices] = {};

// First call on a device (with that device current): resolve the device
// address of the static array once and cache it.
int partials_for_current_device (double **out)
{
  int dev = -1;
  if (cudaGetDevice (&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return FDTD_ERR_CUDA;
  std::lock_guard<std::mutex> lock (g_setup_mutex);
  if (!g_partials_addr[dev])
  {
    void *ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress (&ptr, g_noalloc_partials);
    if (e != cudaSuccess || !ptr)
      return FDTD_ERR_CUDA;
    g_partials_addr[dev] = (double *) ptr;
  }
  *out = g_partials_addr[dev];
  return FDTD_OK;
}

}  // namespace

}  // namespace fdtdb

extern "C" int fdtd_reduce_sq_noalloc (const void *src, int src_kind, size_t n, const void *weight, int weight_kind,
                                       double scale, int blocks, double *out_dev, void *stream)
{
  using namespace fdtdb;
  if (!out_dev || (n > 0 && !src) || src_kind < 0 || src_kind > 2 || weight_kind < 0 || weight_kind > 2
      || (weight_kind != 0 && !weight) || blocks < 0)
    return FDTD_ERR_ARG;
  if (blocks > kNoAllocMaxBlocks)
    return FDTD_ERR_ARG;   // more partials than the static scratch holds
  if (blocks == 0)
  {
    size_t want = (n + 255) / 256;
    blocks = (int) (want < 1 ? 1 : (want > (size_t) kNoAllocMaxBlocks ? kNoAllocMaxBlocks : want));
  }
  double *partials = nullptr;
  int r = partials_for_current_device (&partials);
  if (r != FDTD_OK)
    return r;
  cudaStream_t s = (cudaStream_t) stream;
  launch_reduce_sq (src, src_kind, n, weight, weight_kind, scale, partials, blocks, s);
  launch_reduce_final (partials, blocks, out_dev, s);
  return cudaGetLastError () == cudaSuccess ? FDTD_OK : FDTD_ERR_CUDA;
}
