// ntff.cu - near-to-far-field surface sums (3-D), one kernel over every face
// point of the box and every azimuth, then an ordered reduction.
//
// Per face point the terms are those of the reference's ntffN3D_x/y/z (H on
// the face, averaged over the current and the previous time level) and
// ntffL3D_x/y/z (E on the face, current level), with their sample positions
// per layout, including the H_CENTERED z faces that take the first component
// twice at -1/2 (Source/Scheme/SchemeHelper.h:1036-2095), the phase exponent
// exp(i k r.u) about the grid centre n / 2, and the face signs.  Complex
// arithmetic is the reference's CComplex: products with a real scale
// component-wise, products of two complex values in full.
#include <cuda_fp16.h>

#include "ntff.h"

namespace fdtdb {

namespace {

struct Cx
{
  double re, im;
};

__device__ __forceinline__ Cx operator+ (Cx a, Cx b)
{
  return {a.re + b.re, a.im + b.im};
}
__device__ __forceinline__ Cx operator- (Cx a)
{
  return {-a.re, -a.im};
}
__device__ __forceinline__ Cx operator* (Cx a, double s)
{
  return {a.re * s, a.im * s};
}
__device__ __forceinline__ Cx operator/ (Cx a, double s)
{
  return {a.re / s, a.im / s};
}
__device__ __forceinline__ Cx operator* (Cx a, Cx b)
{
  return {a.re * b.re - a.im * b.im, a.im * b.re + a.re * b.im};
}

enum { EX, EY, EZ, HX, HY, HZ };

// Cell of a position relative to the component's first position (integer
// valued by construction; the reference's convertCoord truncates).  Clamped
// into the grid as a guard; the host checks the box so that it never acts.
__device__ __forceinline__ int64_t cell (const NtffParams &p, const double q[3])
{
  int i[3];
#pragma unroll
  for (int a = 0; a < 3; ++a)
    i[a] = min (max ((int) q[a], 0), p.n[a] - 1);
  return ((int64_t) i[0] * p.n[1] + i[1]) * p.n[2] + i[2];
}

// A stored field value in physical units (FP64 as stored; FP32 / FP16
// storage converted and scaled: H is kept as eta0 H there)
__device__ __forceinline__ double fval (const NtffParams &p, const void *a, int c, int64_t id)
{
  if (p.kind == 0)
    return static_cast<const double *> (a)[id];
  if (p.kind == 1)
    return (double) static_cast<const float *> (a)[id] * p.scale[c];
  return (double) __half2float (static_cast<const __half *> (a)[id]) * p.scale[c];
}
__device__ __forceinline__ Cx cur (const NtffParams &p, int c, int64_t id)
{
  return {fval (p, p.cur[0][c], c, id), fval (p, p.cur[1][c], c, id)};
}
__device__ __forceinline__ Cx prev (const NtffParams &p, int c, int64_t id)
{
  return {fval (p, p.prev[0][c], c, id), fval (p, p.prev[1][c], c, id)};
}

// Component c at position x: one cell, or the two cells at -/+ 1/2 along
// avg_axis; over the two time levels when tavg.
__device__ Cx sample (const NtffParams &p, int c, const double x[3], int avg_axis, bool tavg)
{
  double q[3];
#pragma unroll
  for (int a = 0; a < 3; ++a)
    q[a] = x[a] - p.min_fp[c][a];
  if (avg_axis < 0)
  {
    const int64_t id = cell (p, q);
    return tavg ? (cur (p, c, id) + prev (p, c, id)) / 2.0 : cur (p, c, id);
  }
  double q1[3] = {q[0], q[1], q[2]}, q2[3] = {q[0], q[1], q[2]};
  q1[avg_axis] -= 0.5;
  q2[avg_axis] += 0.5;
  const int64_t i1 = cell (p, q1), i2 = cell (p, q2);
  if (tavg)
    return (cur (p, c, i1) + cur (p, c, i2) + prev (p, c, i1) + prev (p, c, i2)) / 4.0;
  return (cur (p, c, i1) + cur (p, c, i2)) / 2.0;
}

// The two samples of a face term: "first" at -/+ 1/2 along axis b (E_CENTERED)
// or c (H_CENTERED), "second" along the other tangential axis.
struct Pair
{
  Cx a, b;   // (A1 + A2) / 2, (B1 + B2) / 2
};

__device__ Pair face_pair (const NtffParams &p, const double x[3], int axis, int ca, int cb, bool n_sum)
{
  // tangential axes in increasing order
  const int tb = axis == 0 ? 1 : 0;
  const int tc = axis == 2 ? 1 : 2;
  const bool hc = p.h_centered != 0;
  // which fields sit off the face and average across it: H of the N sums in
  // H_CENTERED, E of the L sums in E_CENTERED
  const int avg = (n_sum == hc) ? axis : -1;
  const int sa = hc ? tc : tb;   // axis of the "first" pair
  const int sb = hc ? tb : tc;   // axis of the "second" pair
  double a1[3] = {x[0], x[1], x[2]}, a2[3] = {x[0], x[1], x[2]};
  double b1[3] = {x[0], x[1], x[2]}, b2[3] = {x[0], x[1], x[2]};
  a1[sa] -= 0.5;
  // H_CENTERED z faces: the reference samples the first component twice at
  // -1/2 (SchemeHelper.h ntffN3D_z / ntffL3D_z)
  a2[sa] += (hc && axis == 2) ? -0.5 : 0.5;
  b1[sb] -= 0.5;
  b2[sb] += 0.5;
  Pair r;
  r.a = (sample (p, ca, a1, avg, n_sum) + sample (p, ca, a2, avg, n_sum)) / 2.0;
  r.b = (sample (p, cb, b1, avg, n_sum) + sample (p, cb, b2, avg, n_sum)) / 2.0;
  return r;
}

__global__ void __launch_bounds__ (256) ntff_kernel (NtffParams p, const double *phi, double *partial)
{
  const int ia = blockIdx.y;
  const double ang = phi[ia];
  const double st = sin (p.teta), ct = cos (p.teta);
  const double sp = sin (ang), cp = cos (ang);
  const int L[3] = {p.right[0] - p.left[0], p.right[1] - p.left[1], p.right[2] - p.left[2]};
  const int64_t fx = (int64_t) L[1] * L[2], fy = (int64_t) L[0] * L[2], fz = (int64_t) L[0] * L[1];
  const double d2 = p.dx * p.dx;
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < p.points; i += (int64_t) gridDim.x * blockDim.x)
  {
    // faces: x left, x right, y left, y right, z left, z right
    int64_t r = i;
    int axis, side;
    if (r < 2 * fx)
    {
      axis = 0;
      side = (int) (r / fx);
      r %= fx;
    }
    else if ((r -= 2 * fx) < 2 * fy)
    {
      axis = 1;
      side = (int) (r / fy);
      r %= fy;
    }
    else
    {
      r -= 2 * fy;
      axis = 2;
      side = (int) (r / fz);
      r %= fz;
    }
    const int tb = axis == 0 ? 1 : 0;
    const int tc = axis == 2 ? 1 : 2;
    double x[3];
    x[axis] = side ? p.right[axis] : p.left[axis];
    x[tb] = p.left[tb] + 0.5 + (double) (r / L[tc]);
    x[tc] = p.left[tc] + 0.5 + (double) (r % L[tc]);
    const double s = side ? 1.0 : -1.0;

    double arg = (x[0] - p.diff0[0]) * st * cp + (x[1] - p.diff0[1]) * st * sp + (x[2] - p.diff0[2]) * ct;
    arg *= p.dx;
    const Cx e = {cos (p.k * arg), sin (p.k * arg)};

    Cx nt, np, lt, lp;
    if (axis == 0)
    {
      const Pair n = face_pair (p, x, 0, HZ, HY, true);
      const Pair l = face_pair (p, x, 0, EY, EZ, false);
      nt = (n.a * ct * sp + n.b * st) * e * d2 * -1.0 * s;
      np = (n.a * cp) * e * d2 * -1.0 * s;
      lt = (l.b * ct * sp + l.a * st) * e * d2 * s;
      lp = (l.b * cp) * e * d2 * s;
    }
    else if (axis == 1)
    {
      const Pair n = face_pair (p, x, 1, HZ, HX, true);
      const Pair l = face_pair (p, x, 1, EX, EZ, false);
      nt = (n.a * ct * cp + n.b * st) * e * d2 * s;
      np = (n.a * sp) * e * d2 * -1.0 * s;
      lt = (l.b * ct * cp + l.a * st) * e * d2 * -1.0 * s;
      lp = (l.b * sp) * e * d2 * s;
    }
    else
    {
      const Pair n = face_pair (p, x, 2, HY, HX, true);
      const Pair l = face_pair (p, x, 2, EX, EY, false);
      nt = (-n.a * ct * cp + n.b * ct * sp) * e * d2 * s;
      np = (n.a * sp + n.b * cp) * e * d2 * s;
      lt = (l.b * ct * cp + -l.a * ct * sp) * e * d2 * s;
      lp = (l.b * sp + l.a * cp) * e * d2 * -1.0 * s;
    }
    acc[0] += nt.re;
    acc[1] += nt.im;
    acc[2] += np.re;
    acc[3] += np.im;
    acc[4] += lt.re;
    acc[5] += lt.im;
    acc[6] += lp.re;
    acc[7] += lp.im;
  }
  __shared__ double red[8][256];
#pragma unroll
  for (int j = 0; j < 8; ++j)
    red[j][threadIdx.x] = acc[j];
  __syncthreads ();
  for (int w = blockDim.x / 2; w > 0; w >>= 1)
  {
    if ((int) threadIdx.x < w)
    {
#pragma unroll
      for (int j = 0; j < 8; ++j)
        red[j][threadIdx.x] += red[j][threadIdx.x + w];
    }
    __syncthreads ();
  }
  if (threadIdx.x < 8)
    partial[((int64_t) ia * gridDim.x + blockIdx.x) * 8 + threadIdx.x] = red[threadIdx.x][0];
}

// Sums the per-block partials of every azimuth in block order.
__global__ void ntff_final_kernel (const double *partial, int blocks, int nphi, double *out)
{
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nphi * 8)
    return;
  const int ia = t / 8, j = t % 8;
  double s = 0.0;
  for (int b = 0; b < blocks; ++b)
    s += partial[((int64_t) ia * blocks + b) * 8 + j];
  out[t] = s;
}

}  // namespace

int launch_ntff (const NtffParams &p, const double *phi_dev, int nphi, double *partial, int blocks, double *out,
                 cudaStream_t s)
{
  ntff_kernel<<<dim3 ((unsigned) blocks, (unsigned) nphi), 256, 0, s>>> (p, phi_dev, partial);
  ntff_final_kernel<<<(nphi * 8 + 255) / 256, 256, 0, s>>> (partial, blocks, nphi, out);
  return 2;
}

}  // namespace fdtdb
