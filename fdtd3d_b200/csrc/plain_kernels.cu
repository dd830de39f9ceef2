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
// * fine_average_kernel: double material precision - one component's
//   material, averaged over the eight fine cells around it
//   (YeeGridLayout.h:866-1030, Approximation.cpp:34-54), once per upload.
#include <cuda_runtime.h>

#include "kernels.h"
#include "plain_cell.cuh"

namespace fdtdb {

template <bool DMP, bool CS>
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
#pragma unroll
    for (int ci = 0; ci < 3; ++ci)
    {
      if (p.comp[ci].exists)
        plain_component<DMP, CS> (p, ci, inc_len, err, x, y, z);
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
  if (p.dmp)
  {
    if (p.cs_mask)
      plain_half_kernel<true, true><<<(unsigned) blocks, 256, 0, s>>> (p, inc_len, err);
    else
      plain_half_kernel<true, false><<<(unsigned) blocks, 256, 0, s>>> (p, inc_len, err);
  }
  else if (p.cs_mask)
    plain_half_kernel<false, true><<<(unsigned) blocks, 256, 0, s>>> (p, inc_len, err);
  else
    plain_half_kernel<false, false><<<(unsigned) blocks, 256, 0, s>>> (p, inc_len, err);
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

__global__ void fine_average_kernel (const double *fine, double *out64, float *out32, FineAvg a)
{
  const int64_t total = (int64_t) a.n[0] * a.n[1] * a.n[2];
  for (int64_t id = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; id < total;
       id += (int64_t) gridDim.x * blockDim.x)
  {
    const int z = (int) (id % a.n[2]);
    const int64_t r = id / a.n[2];
    const int y = (int) (r % a.n[1]);
    const int x = (int) (r / a.n[1]);
    const int p[3] = {x, y, z};
    double v[8];
#pragma unroll
    for (int j = 0; j < 8; ++j)
    {
      // the outer shell's last cell would reach one fine cell past the grid;
      // its material is never used, so clamp
      int q[3];
#pragma unroll
      for (int b = 0; b < 3; ++b)
        q[b] = min (a.mul[b] * p[b] + a.off[j][b], a.nf[b] - 1);
      v[j] = fine[((int64_t) q[0] * a.nf[1] + q[1]) * a.nf[2] + q[2]];
    }
    // ((v1 + v2) / 2 + (v3 + v4) / 2) / 2, twice, then / 2
    const double lo = ((v[0] + v[1]) / 2.0 + (v[2] + v[3]) / 2.0) / 2.0;
    const double hi = ((v[4] + v[5]) / 2.0 + (v[6] + v[7]) / 2.0) / 2.0;
    const double m = (lo + hi) / 2.0;
    if (out64)
      out64[id] = m;
    if (out32)
      out32[id] = (float) m;
  }
}

// Scattered field for a dump (Scheme::makeGridScattered, Source/Scheme/
// Scheme.inc.h:4113-4226): inside the TF/SF box (real coordinates within
// [left, right] on every kept axis) the component minus its incident value.
__global__ void scattered_kernel (double *f, GeomDev g, int k, const double *inc, int inc_len, double3 left,
                                  double3 right, int *err)
{
  const int64_t total = (int64_t) g.n[0] * g.n[1] * g.n[2];
  const double lo[3] = {left.x, left.y, left.z}, hi[3] = {right.x, right.y, right.z};
  for (int64_t id = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; id < total;
       id += (int64_t) gridDim.x * blockDim.x)
  {
    const int z = (int) (id % g.n[2]);
    const int64_t r = id / g.n[2];
    const int y = (int) (r % g.n[1]);
    const int x = (int) (r / g.n[1]);
    const int p[3] = {x, y, z};
    bool inside = true;
#pragma unroll
    for (int a = 0; a < 3; ++a)
    {
      const double c = (double) p[a] + g.min_fp[k][a];
      if (!((g.drop >> a) & 1) && (c < lo[a] || c > hi[a]))
        inside = false;
    }
    if (inside)
      f[id] = f[id] - incident_value (g, inc, inc_len, err, k, x, y, z);
  }
}

int launch_scattered (double *f, const GeomDev &g, int k, const double *inc, int inc_len, const double left[3],
                      const double right[3], int *err, int sm_count, cudaStream_t s)
{
  scattered_kernel<<<sm_count * 4, 256, 0, s>>> (f, g, k, inc, inc_len, make_double3 (left[0], left[1], left[2]),
                                                 make_double3 (right[0], right[1], right[2]), err);
  return 1;
}

int launch_fine_average (const double *fine, double *out64, float *out32, const FineAvg &a, int sm_count,
                         cudaStream_t s)
{
  fine_average_kernel<<<sm_count * 4, 256, 0, s>>> (fine, out64, out32, a);
  return 1;
}

}  // namespace fdtdb
