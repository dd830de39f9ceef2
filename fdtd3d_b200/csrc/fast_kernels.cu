// fast_kernels.cu - FP32 / FP16-storage form of the fdtd3d step, plus the
// conversion and reduction kernels.
//
// Formulation (algebraically the reference's, re-scaled and with the PML
// auxiliary fields kept only where sigma != 0):
//   H is stored as H' = eta0 * H, so with S = c*dt/dx every update reads
//     interior cells:  F += S / m * curl
//     PML cells:       X_new = ca1 * X + S * q1 * curl
//                      F     = p5 * F + (g4p * X_new - g4m * X) * q5 / m
//   where m is the averaged eps (E) or mu (H), X = D/eps0 or c*B, and the
//   1-D tables come from the reference's sigma profiles
//   (Source/Scheme/InternalScheme.inc.h:2297-2349, 2551-2640; the PML
//   coefficients of H use eps0 as in the reference).  In interior cells the
//   reference's D/B chain with sigma = 0 reduces exactly to the first line.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "cell_walk.cuh"
#include "kernels.h"

namespace fdtdb {

namespace {

template <typename T>
__device__ __forceinline__ float ld (const T *p, size_t i);
template <>
__device__ __forceinline__ float ld<float> (const float *p, size_t i)
{
  return p[i];
}
template <>
__device__ __forceinline__ float ld<__half> (const __half *p, size_t i)
{
  return __half2float (p[i]);
}

template <typename T>
__device__ __forceinline__ void st (T *p, size_t i, float v);
template <>
__device__ __forceinline__ void st<float> (float *p, size_t i, float v)
{
  p[i] = v;
}
template <>
__device__ __forceinline__ void st<__half> (__half *p, size_t i, float v)
{
  p[i] = __float2half_rn (v);
}

__device__ __forceinline__ size_t flin (const GeomDev &g, int x, int y, int z)
{
  return ((size_t) x * g.n[1] + y) * g.n[2] + z;
}

// incident value in FP64 (1-D grid is FP64 in every form)
__device__ __forceinline__ double fast_incident (const GeomDev &g, const double *inc, int inc_len, int *err, int k,
                                                 int px, int py, int pz)
{
  double d_diff = k >= 3 ? 0.5 : 0.0;
  double d;
  const int pos[3] = {px, py, pz};
  if (g.drop == 0)
  {
    double x = ((double) px + g.min_fp[k][0]) - g.zero_inc[0];
    double y = ((double) py + g.min_fp[k][1]) - g.zero_inc[1];
    double z = ((double) pz + g.min_fp[k][2]) - g.zero_inc[2];
    d = x * g.s1 * g.c2 + y * g.s1 * g.s2 + z * g.c1 - d_diff;
  }
  else
  {
    const int a0 = g.inc_ax[0], a1 = g.inc_ax[1];
    double u = ((double) pos[a0] + g.min_fp[k][a0]) - g.zero_inc[a0];
    double v = ((double) pos[a1] + g.min_fp[k][a1]) - g.zero_inc[a1];
    d = u * g.inc_k[0] + v * g.inc_k[1] - d_diff;
  }
  int i1 = (int) d;
  double pr2 = d - (double) i1;
  if (i1 < 0 || i1 + 1 >= inc_len)
  {
    if (err)
      *err = 1;
    return 0.0;
  }
  return (inc[i1] * (1 - pr2) + inc[i1 + 1] * pr2) * g.proj[k];
}

template <typename T>
__device__ __forceinline__ void fast_component (const FastHalf &p, int ci, int *err, int x, int y, int z)
{
  const GeomDev &g = p.g;
  const CompDev &c = p.comp[ci];
  const size_t id = flin (g, x, y, z);
  T *F = (T *) p.f[ci];
  const T *o1 = (const T *) p.opp[c.opp1];
  const T *o2 = (const T *) p.opp[c.opp2];
  float v0 = 0.f, v1 = 0.f, v2 = 0.f, v3 = 0.f;
  if (o1)
  {
    v0 = ld (o1, flin (g, x + c.d11[0], y + c.d11[1], z + c.d11[2]));
    v1 = ld (o1, flin (g, x + c.d12[0], y + c.d12[1], z + c.d12[2]));
  }
  if (o2)
  {
    v2 = ld (o2, flin (g, x + c.d21[0], y + c.d21[1], z + c.d21[2]));
    v3 = ld (o2, flin (g, x + c.d22[0], y + c.d22[1], z + c.d22[2]));
  }
  if (p.use_tfsf)
  {
    for (int t = 0; t < c.nterms; ++t)
    {
      const TermDev &tm = c.term[t];
      if (x >= tm.lo[0] && x < tm.hi[0] && y >= tm.lo[1] && y < tm.hi[1] && z >= tm.lo[2] && z < tm.hi[2])
      {
        double diff = fast_incident (g, p.inc, p.inc_len, err, tm.inc_comp, x + tm.aux[0], y + tm.aux[1],
                                     z + tm.aux[2]);
        float dv = (float) (diff * tm.negate) * p.inc_scale[tm.inc_comp];
        if (tm.slot == 0)
          v0 -= dv;
        else if (tm.slot == 1)
          v1 -= dv;
        else if (tm.slot == 2)
          v2 -= dv;
        else
          v3 -= dv;
      }
    }
  }
  float curl = (v1 - v0) - (v3 - v2);
  // J / M current source: the reference subtracts I dx Cb from the new D
  // (or E), i.e. I dx from the curl, here in the curl's scaled units
  if (((p.cs_mask >> ci) & 1) && x == p.cs[0] && y == p.cs[1] && z == p.cs[2])
    curl -= (float) (*p.cs_val * p.g.dx) * p.cs_scale;

  float inv_m = 1.f, m = 1.f;
  const float *mp = p.matc[ci] ? p.matc[ci] : p.mat;
  if (mp)
  {
    if (c.nmat == 1)
      m = mp[id];
    else if (c.nmat == 2)
      m = 0.5f * (mp[flin (g, x, y, z)] + mp[flin (g, x + c.m[1][0], y + c.m[1][1], z + c.m[1][2])]);
    else
      m = 0.25f * (mp[flin (g, x, y, z)] + mp[flin (g, x + c.m[1][0], y + c.m[1][1], z + c.m[1][2])]
                   + mp[flin (g, x + c.m[2][0], y + c.m[2][1], z + c.m[2][2])]
                   + mp[flin (g, x + c.m[3][0], y + c.m[3][1], z + c.m[3][2])]);
    inv_m = 1.f / m;
  }

  const int pos[3] = {x, y, z};
  bool interior = true;
  if (p.use_pml)
  {
#pragma unroll
    for (int a = 0; a < 3; ++a)
      interior = interior && pos[a] >= p.ilo[ci][a] && pos[a] < p.ihi[ci][a];
  }
  float f = ld (F, id);
  // Drude cell: a nonzero plasma frequency or collision rate on the
  // component's averaging stencil (getMetaMaterial: the mean of its two or
  // four points; metamaterials run with PML, as the reference's do)
  float w = 0.f, gm = 0.f;
  if (p.meta)
  {
    for (int j = 0; j < c.nmat; ++j)
    {
      const size_t q = flin (g, x + c.m[j][0], y + c.m[j][1], z + c.m[j][2]);
      w += p.om[q];
      gm += p.ga[q];
    }
    const float inv_n = c.nmat == 4 ? 0.25f : (c.nmat == 2 ? 0.5f : 1.f);
    w *= inv_n;
    gm *= inv_n;
  }
  if (p.meta && (w != 0.f || gm != 0.f))
  {
    // X by the curl step (PML coefficients; sigma = 0 gives ca1 = 1,
    // sq1 = S), the Drude recurrence to Z (the reference's b0 .. a2,
    // InternalScheme.inc.h:2527-2532, in the scaled units), F from Z with
    // material modifier 1 (InternalScheme.inc.h:2452-2640).  The recurrence
    // Z_n = b0 X_n + b1 X_o + b2 X_pp - a1 Z_o - a2 Z_pp is evaluated on
    // increments (b0 + b1 + b2 = 0 and 1 + a1 + a2 = 4 sq / A):
    //   dZ = b0 dX - b2 dX_o + a2 dZ_o - (4 sq / A) Z_o,
    // so that FP32 does not subtract nearly equal products of the fields;
    // this path keeps the last increments dX_o, dZ_o per cell (xpp, zpp).
    const int a0 = c.sig4, a1 = c.sig_cacb, a2 = c.sig5;
    const float ca1 = p.tab[ci][0][pos[a1]];
    const float sq1 = p.tab[ci][1][pos[a1]];
    const float p5 = p.tab[ci][2][pos[a2]];
    const float q5 = p.tab[ci][3][pos[a2]];
    const float g4p = p.tab[ci][4][pos[a0]];
    const float g4m = p.tab[ci][5][pos[a0]];
    float *X = p.aux[ci];
    const float xo = X[id], dxo = p.xpp[ci][id], zo = p.zd[ci][id], dzo = p.zpp[ci][id];
    const float dt = p.dt;
    const float sq = (dt * w) * (dt * w);
    const float inv = 1.f / (4.f * m + 2.f * dt * m * gm + sq);
    const float b0 = (4.f + 2.f * dt * gm) * inv, b2 = (4.f - 2.f * dt * gm) * inv;
    const float a2c = (4.f * m - 2.f * dt * m * gm + sq) * inv;
    const float dx = (ca1 - 1.f) * xo + sq1 * curl;
    const float dz = b0 * dx - b2 * dxo + a2c * dzo - (4.f * sq * inv) * zo;
    X[id] = xo + dx;
    p.xpp[ci][id] = dx;
    p.zd[ci][id] = zo + dz;
    p.zpp[ci][id] = dz;
    f = p5 * f + ((g4p - g4m) * zo + g4p * dz) * q5;
  }
  else if (interior)
  {
    f += p.courant * inv_m * curl;
  }
  else
  {
    const int a0 = c.sig4, a1 = c.sig_cacb, a2 = c.sig5;
    const float ca1 = p.tab[ci][0][pos[a1]];
    const float sq1 = p.tab[ci][1][pos[a1]];
    const float p5 = p.tab[ci][2][pos[a2]];
    const float q5 = p.tab[ci][3][pos[a2]];
    const float g4p = p.tab[ci][4][pos[a0]];
    const float g4m = p.tab[ci][5][pos[a0]];
    float *X = p.aux[ci];
    const float xo = X[id];
    const float xn = ca1 * xo + sq1 * curl;
    X[id] = xn;
    f = p5 * f + (g4p * xn - g4m * xo) * q5 * inv_m;
  }
  st (F, id, f);
}

template <typename T>
__global__ void __launch_bounds__ (256) fast_half_kernel (FastHalf p, int *err)
{
  // interior cells: 1 .. n - 2 on every axis a mode keeps, 0 on a dropped one
  const int ix = (p.g.drop & 1) ? 1 : p.g.n[0] - 2;
  const int iy = (p.g.drop & 2) ? 1 : p.g.n[1] - 2;
  const int iz = (p.g.drop & 4) ? 1 : p.g.n[2] - 2;
  const int oz = (p.g.drop & 4) ? 0 : 1, oy = (p.g.drop & 2) ? 0 : 1, ox = (p.g.drop & 1) ? 0 : 1;
  for (CellWalk w ((int64_t) blockIdx.x * blockDim.x + threadIdx.x, (int64_t) gridDim.x * blockDim.x, ix, iy, iz);
       w.ok (); w.next ())
  {
    const int z = w.cz + oz, y = w.cy + oy, x = w.cx + ox;
#pragma unroll 1
    for (int ci = 0; ci < 3; ++ci)
    {
      if (p.comp[ci].exists)
        fast_component<T> (p, ci, err, x, y, z);
    }
  }
}

template <typename T>
__global__ void fast_point_source_kernel (T *f, size_t index, const double *src, int src_index, float scale)
{
  if (threadIdx.x == 0 && blockIdx.x == 0)
    st (f, index, (float) src[src_index] * scale);
}

template <typename T>
__global__ void convert_in_kernel (T *dst, const double *src, size_t n, double scale)
{
  for (size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t) gridDim.x * blockDim.x)
    st (dst, i, (float) (src[i] * scale));
}

__global__ void convert_in_double_kernel (double *dst, const double *src, size_t n, double scale)
{
  for (size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t) gridDim.x * blockDim.x)
    dst[i] = src[i] * scale;
}

template <typename T>
__global__ void convert_out_kernel (double *dst, const T *src, size_t n, double scale)
{
  for (size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t) gridDim.x * blockDim.x)
    dst[i] = (double) ld (src, i) * scale;
}

__global__ void convert_out_double_kernel (double *dst, const double *src, size_t n, double scale)
{
  for (size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t) gridDim.x * blockDim.x)
    dst[i] = src[i] * scale;
}

// Neumaier (compensated) accumulation in FP64
__device__ __forceinline__ void neumaier (double &s, double &c, double v)
{
  double t = s + v;
  if (fabs (s) >= fabs (v))
    c += (s - t) + v;
  else
    c += (v - t) + s;
  s = t;
}

template <typename T>
__device__ __forceinline__ double ldd (const void *p, size_t i)
{
  return (double) ld ((const T *) p, i);
}

template <int KIND>
__global__ void __launch_bounds__ (256) reduce_sq_kernel (const void *src, size_t n, const void *weight,
                                                          int wkind, double scale, double *partials)
{
  double s = 0.0, c = 0.0;
  for (size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t) gridDim.x * blockDim.x)
  {
    double v;
    if (KIND == 0)
      v = ((const double *) src)[i];
    else if (KIND == 1)
      v = ldd<float> (src, i);
    else
      v = ldd<__half> (src, i);
    double w = 1.0;
    if (wkind == 1)
      w = (double) ((const float *) weight)[i];
    else if (wkind == 2)
      w = ((const double *) weight)[i];
    neumaier (s, c, w * v * v * scale);
  }
  __shared__ double ss[256];
  __shared__ double sc[256];
  ss[threadIdx.x] = s;
  sc[threadIdx.x] = c;
  __syncthreads ();
  if (threadIdx.x == 0)
  {
    double bs = 0.0, bc = 0.0;
    for (int i = 0; i < blockDim.x; ++i)
    {
      neumaier (bs, bc, ss[i]);
      bc += sc[i];
    }
    partials[2 * blockIdx.x] = bs;
    partials[2 * blockIdx.x + 1] = bc;
  }
}

__global__ void reduce_final_kernel (const double *partials, int nblocks, double *out)
{
  if (threadIdx.x == 0 && blockIdx.x == 0)
  {
    double s = 0.0, c = 0.0;
    for (int i = 0; i < nblocks; ++i)
    {
      neumaier (s, c, partials[2 * i]);
      c += partials[2 * i + 1];
    }
    out[0] = s + c;
  }
}

int grid_for (size_t n, int sm_count)
{
  size_t b = (n + 255) / 256;
  size_t cap = (size_t) sm_count * 16;
  if (b > cap)
    b = cap;
  return b < 1 ? 1 : (int) b;
}

}  // namespace

int launch_fast_half (const FastHalf &p, int *err, int sm_count, cudaStream_t s)
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
  if (p.fp16)
    fast_half_kernel<__half><<<(unsigned) blocks, 256, 0, s>>> (p, err);
  else
    fast_half_kernel<float><<<(unsigned) blocks, 256, 0, s>>> (p, err);
  return 1;
}

int launch_fast_point_source (void *f, int fp16, size_t index, const double *src, int src_index, float scale,
                              cudaStream_t s)
{
  if (fp16)
    fast_point_source_kernel<__half><<<1, 32, 0, s>>> ((__half *) f, index, src, src_index, scale);
  else
    fast_point_source_kernel<float><<<1, 32, 0, s>>> ((float *) f, index, src, src_index, scale);
  return 1;
}

int launch_convert_in (void *dst, int dst_kind, const double *src, size_t n, double scale, cudaStream_t s)
{
  int blocks = grid_for (n, 148);
  if (dst_kind == 0)
    convert_in_double_kernel<<<blocks, 256, 0, s>>> ((double *) dst, src, n, scale);
  else if (dst_kind == 1)
    convert_in_kernel<float><<<blocks, 256, 0, s>>> ((float *) dst, src, n, scale);
  else
    convert_in_kernel<__half><<<blocks, 256, 0, s>>> ((__half *) dst, src, n, scale);
  return 1;
}

namespace {

// lowest index of a non-finite value (NaN or +-Inf) into *first
__global__ void find_nonfinite_kernel (const double *src, size_t n, unsigned long long *first)
{
  for (size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t) gridDim.x * blockDim.x)
    if (!isfinite (src[i]))
      atomicMin (first, (unsigned long long) i);
}

}  // namespace

int launch_find_nonfinite (const double *src, size_t n, unsigned long long *first, cudaStream_t s)
{
  find_nonfinite_kernel<<<grid_for (n, 148), 256, 0, s>>> (src, n, first);
  return 1;
}

int launch_convert_out (double *dst, const void *src, int src_kind, size_t n, double scale, cudaStream_t s)
{
  int blocks = grid_for (n, 148);
  if (src_kind == 0)
    convert_out_double_kernel<<<blocks, 256, 0, s>>> (dst, (const double *) src, n, scale);
  else if (src_kind == 1)
    convert_out_kernel<float><<<blocks, 256, 0, s>>> (dst, (const float *) src, n, scale);
  else
    convert_out_kernel<__half><<<blocks, 256, 0, s>>> (dst, (const __half *) src, n, scale);
  return 1;
}

int launch_reduce_sq (const void *src, int kind, size_t n, const void *weight, int wkind, double scale,
                      double *partials, int nblocks, cudaStream_t s)
{
  if (kind == 0)
    reduce_sq_kernel<0><<<nblocks, 256, 0, s>>> (src, n, weight, wkind, scale, partials);
  else if (kind == 1)
    reduce_sq_kernel<1><<<nblocks, 256, 0, s>>> (src, n, weight, wkind, scale, partials);
  else
    reduce_sq_kernel<2><<<nblocks, 256, 0, s>>> (src, n, weight, wkind, scale, partials);
  return 1;
}

__global__ void fill_kernel (double *dst, size_t n, double value)
{
  for (size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t) gridDim.x * blockDim.x)
    dst[i] = value;
}

int launch_fill (double *dst, size_t n, double value, cudaStream_t s)
{
  fill_kernel<<<grid_for (n, 148), 256, 0, s>>> (dst, n, value);
  return 1;
}

int launch_reduce_final (const double *partials, int nblocks, double *out, cudaStream_t s)
{
  reduce_final_kernel<<<1, 32, 0, s>>> (partials, nblocks, out);
  return 1;
}

// The same two launches through cudaLaunchKernel, so that each returns its
// own launch status and an earlier, unrelated error pending on the calling
// thread is neither reported nor cleared.
cudaError_t launch_reduce_sq_checked (const void *src, int kind, size_t n, const void *weight, int wkind,
                                      double scale, double *partials, int nblocks, cudaStream_t s)
{
  const void *fn = kind == 0 ? (const void *) reduce_sq_kernel<0>
                   : kind == 1 ? (const void *) reduce_sq_kernel<1>
                               : (const void *) reduce_sq_kernel<2>;
  void *args[] = {(void *) &src, (void *) &n, (void *) &weight, (void *) &wkind, (void *) &scale,
                  (void *) &partials};
  return cudaLaunchKernel (fn, dim3 (nblocks), dim3 (256), args, 0, s);
}

cudaError_t launch_reduce_final_checked (const double *partials, int nblocks, double *out, cudaStream_t s)
{
  void *args[] = {(void *) &partials, (void *) &nblocks, (void *) &out};
  return cudaLaunchKernel ((const void *) reduce_final_kernel, dim3 (1), dim3 (32), args, 0, s);
}

}  // namespace fdtdb

// ------------------------------------------------------------ running DFT

namespace fdtdb {

namespace {

__device__ __forceinline__ double ldd (const double *p, size_t i)
{
  return p[i];
}
__device__ __forceinline__ double ldd (const float *p, size_t i)
{
  return (double) p[i];
}
__device__ __forceinline__ double ldd (const __half *p, size_t i)
{
  return (double) __half2float (p[i]);
}

__device__ __forceinline__ void neumaier (double *s, double *c, double v)
{
  const double t = *s + v;
  if (fabs (*s) >= fabs (v))
    *c += (*s - t) + v;
  else
    *c += (v - t) + *s;
  *s = t;
}

// One time step of the running DFT of a stored field on the plane
// x_axis = index: for every plane cell and frequency j,
//   sum_j += v * exp(-i phase_j),  phase table = (cos, sin) per frequency,
// in FP64 with Neumaier compensation (acc: re, re compensation, im, im
// compensation per cell and frequency).
template <typename T>
__global__ void dft_kernel (const T *src, int axis, int index, int n0, int n1, int n2, double scale,
                            const double *phase, int nf, double *acc)
{
  const int ma = axis == 0 ? n1 : n0;             // plane extents (first, second remaining axis)
  const int mb = axis == 2 ? n1 : n2;
  const long long cells = (long long) ma * mb;
  for (long long q = (long long) blockIdx.x * blockDim.x + threadIdx.x; q < cells * nf;
       q += (long long) gridDim.x * blockDim.x)
  {
    const int j = (int) (q / cells);
    const long long c = q % cells;
    const int a = (int) (c / mb), b = (int) (c % mb);
    long long id;
    if (axis == 0)
      id = ((long long) index * n1 + a) * n2 + b;
    else if (axis == 1)
      id = ((long long) a * n1 + index) * n2 + b;
    else
      id = ((long long) a * n1 + b) * n2 + index;
    const double v = ldd (src, (size_t) id) * scale;
    double *r = acc + q * 4;
    neumaier (r + 0, r + 1, v * phase[2 * j]);
    neumaier (r + 2, r + 3, -v * phase[2 * j + 1]);
  }
}

}  // namespace

int launch_dft (const void *src, int kind, int axis, int index, const int n[3], double scale, const double *phase,
                int nf, double *acc, int sm_count, cudaStream_t s)
{
  const long long cells = (long long) (axis == 0 ? n[1] : n[0]) * (axis == 2 ? n[1] : n[2]) * nf;
  long long blocks = (cells + 255) / 256;
  if (blocks > (long long) sm_count * 16)
    blocks = (long long) sm_count * 16;
  if (kind == 0)
    dft_kernel<double><<<(unsigned) blocks, 256, 0, s>>> ((const double *) src, axis, index, n[0], n[1], n[2], scale,
                                                          phase, nf, acc);
  else if (kind == 1)
    dft_kernel<float><<<(unsigned) blocks, 256, 0, s>>> ((const float *) src, axis, index, n[0], n[1], n[2], scale,
                                                         phase, nf, acc);
  else
    dft_kernel<__half><<<(unsigned) blocks, 256, 0, s>>> ((const __half *) src, axis, index, n[0], n[1], n[2], scale,
                                                          phase, nf, acc);
  return 1;
}

}  // namespace fdtdb
