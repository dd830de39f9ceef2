// plain_kernels.cu - FP64 kernels compiled with --fmad=false.
//
// * plain_half_kernel: one half-step (all E or all H components) of the FP64
//   plain form, one thread per interior cell, curl -> Drude -> E-from-D fused
//   per cell.  Replaces the reference's per-component
//   calculateFieldStepIterationKernel, ...PMLMetamaterialsKernel and
//   ...PMLKernel launches plus their <<<1,1>>> shiftInTime kernels
//   (Source/Scheme/InternalScheme.inc.h:21-432); time levels rotate as kernel
//   arguments instead.
// * incident_e_kernel / incident_h_kernel: the 1-D auxiliary TF/SF grid
//   (InternalScheme.inc.h:3276-3357), FP64 for every form.
// * point_source_kernel: hard sinusoidal source (InternalScheme.inc.h:2818-2895).
#include <cuda_runtime.h>

#include "kernels.h"
#include "plain_cell.cuh"

namespace fdtdb {

__global__ void __launch_bounds__ (256) plain_half_kernel (PlainHalf p, int inc_len, int *err)
{
  // interior cells: 1 .. n - 2 on every axis a mode keeps, 0 on a dropped one
  const int ix = (p.g.drop & 1) ? 1 : p.g.n[0] - 2;
  const int iy = (p.g.drop & 2) ? 1 : p.g.n[1] - 2;
  const int iz = (p.g.drop & 4) ? 1 : p.g.n[2] - 2;
  const int64_t total = (int64_t) ix * iy * iz;
  for (int64_t tid = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; tid < total;
       tid += (int64_t) gridDim.x * blockDim.x)
  {
    const int z = (int) (tid % iz) + ((p.g.drop & 4) ? 0 : 1);
    const int64_t r = tid / iz;
    const int y = (int) (r % iy) + ((p.g.drop & 2) ? 0 : 1);
    const int x = (int) (r / iy) + ((p.g.drop & 1) ? 0 : 1);
#pragma unroll 1
    for (int ci = 0; ci < 3; ++ci)
    {
      if (p.comp[ci].exists)
        plain_component (p, ci, inc_len, err, x, y, z);
    }
  }
}

__global__ void incident_e_kernel (double *e_new, const double *e_old, const double *h_old, int len,
                                   double modifier, const double *src, int src_index)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < len; i += gridDim.x * blockDim.x)
  {
    if (i == 0)
      e_new[0] = src[src_index];
    else
      e_new[i] = e_old[i] + (h_old[i - 1] - h_old[i]) * modifier;
  }
}

__global__ void incident_h_kernel (double *h_new, const double *h_old, const double *e_new, int len,
                                   double modifier)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < len - 1; i += gridDim.x * blockDim.x)
    h_new[i] = h_old[i] + (e_new[i] - e_new[i + 1]) * modifier;
}

__global__ void point_source_kernel (double *f, size_t index, const double *src, int src_index)
{
  if (threadIdx.x == 0 && blockIdx.x == 0)
    f[index] = src[src_index];
}

int launch_plain_half (const PlainHalf &p, int inc_len, int *err, int sm_count, cudaStream_t s)
{
  const int ix = (p.g.drop & 1) ? 1 : p.g.n[0] - 2;
  const int iy = (p.g.drop & 2) ? 1 : p.g.n[1] - 2;
  const int iz = (p.g.drop & 4) ? 1 : p.g.n[2] - 2;
  int64_t total = (int64_t) ix * iy * iz;
  int64_t blocks = (total + 255) / 256;
  int64_t cap = (int64_t) sm_count * 8 * 16;
  if (blocks > cap)
    blocks = cap;
  if (blocks < 1)
    blocks = 1;
  plain_half_kernel<<<(unsigned) blocks, 256, 0, s>>> (p, inc_len, err);
  return 1;
}

int launch_incident_e (double *e_new, const double *e_old, const double *h_old, int len, double modifier,
                       const double *src, int src_index, cudaStream_t s)
{
  int blocks = (len + 255) / 256;
  incident_e_kernel<<<blocks, 256, 0, s>>> (e_new, e_old, h_old, len, modifier, src, src_index);
  return 1;
}

int launch_incident_h (double *h_new, const double *h_old, const double *e_new, int len, double modifier,
                       cudaStream_t s)
{
  int blocks = (len + 255) / 256;
  incident_h_kernel<<<blocks, 256, 0, s>>> (h_new, h_old, e_new, len, modifier);
  return 1;
}

int launch_point_source (double *f, size_t index, const double *src, int src_index, cudaStream_t s)
{
  point_source_kernel<<<1, 32, 0, s>>> (f, index, src, src_index);
  return 1;
}

}  // namespace fdtdb
