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
// The array is kNoAllocMaxBlocks pairs of doubles (16 KiB).  Every GPU that
// loads the library holds it until the process exits.  All calls share it,
// so calls that overlap on the GPU (different streams, or different host
// threads on one device) race on it and must be ordered by the caller.
// Each call rewrites every partial it reads before reading it, so nothing
// has to be cleared between calls.
#include <cuda_runtime.h>

#include <string>

#include "../../include/fdtd_b200.h"
#include "kernels.h"

namespace fdtdb {

namespace {

constexpr int kNoAllocMaxBlocks = 1024;

// (sum, compensation) per block.  In host code this name is only a
// stand-in for the device array, never a device address: its address on the
// current device comes from cudaGetSymbolAddress.
__device__ __align__ (256) double g_noalloc_partials[2 * kNoAllocMaxBlocks];

int refuse (int code, const std::string &msg)
{
  set_last_error (msg.c_str ());
  return code;
}

// Device address of the static array on the current device.  The first call
// on a device loads the library's device code there (the set-up); later
// calls are a lookup in the runtime's table.  Looking the address up on
// every call (rather than caching it per device ordinal) keeps it right
// after a cudaDeviceReset, which reloads the device code at a new address.
int partials_for_current_device (double **out)
{
  void *ptr = nullptr;
  const cudaError_t e = cudaGetSymbolAddress (&ptr, g_noalloc_partials);
  if (e != cudaSuccess || !ptr)
  {
    if (e != cudaSuccess)
      cudaGetLastError ();   // the failure above is this call's own: do not leave it pending
    return refuse (FDTD_ERR_CUDA, std::string ("cudaGetSymbolAddress of the static scratch: ") +
                                      cudaGetErrorString (e));
  }
  *out = (double *) ptr;
  return FDTD_OK;
}

}  // namespace

}  // namespace fdtdb

extern "C" int fdtd_reduce_sq_noalloc (const void *src, int src_kind, size_t n, const void *weight, int weight_kind,
                                       double scale, int blocks, double *out_dev, void *stream)
{
  using namespace fdtdb;
  if (!out_dev || (n > 0 && !src))
    return refuse (FDTD_ERR_ARG, "fdtd_reduce_sq_noalloc: null output, or null input with n > 0");
  if (src_kind < 0 || src_kind > 2)
    return refuse (FDTD_ERR_ARG, "fdtd_reduce_sq_noalloc: src_kind must be 0 (double), 1 (float) or 2 (half)");
  if (weight_kind < 0 || weight_kind > 2)
    return refuse (FDTD_ERR_ARG, "fdtd_reduce_sq_noalloc: weight_kind must be 0 (none), 1 (float) or 2 (double)");
  if (weight_kind != 0 && !weight)
    return refuse (FDTD_ERR_ARG, "fdtd_reduce_sq_noalloc: weight_kind != 0 needs a weight buffer");
  if (blocks < 0 || blocks > kNoAllocMaxBlocks)
    return refuse (FDTD_ERR_ARG, "fdtd_reduce_sq_noalloc: blocks must be 0 (automatic) .. 1024, the size of the "
                                 "static scratch");
  if (blocks == 0)
  {
    const size_t want = (n + 255) / 256;
    blocks = (int) (want < 1 ? 1 : (want > (size_t) kNoAllocMaxBlocks ? kNoAllocMaxBlocks : want));
  }
  double *partials = nullptr;
  const int r = partials_for_current_device (&partials);
  if (r != FDTD_OK)
    return r;
  const cudaStream_t s = (cudaStream_t) stream;
  cudaError_t e = launch_reduce_sq_checked (src, src_kind, n, weight, weight_kind, scale, partials, blocks, s);
  if (e == cudaSuccess)
    e = launch_reduce_final_checked (partials, blocks, out_dev, s);
  if (e != cudaSuccess)
  {
    cudaGetLastError ();   // clear this call's own launch error
    return refuse (FDTD_ERR_CUDA, std::string ("fdtd_reduce_sq_noalloc: launch failed: ") + cudaGetErrorString (e));
  }
  return FDTD_OK;
}
