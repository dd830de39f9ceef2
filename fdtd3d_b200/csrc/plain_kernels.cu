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

#include "cell_walk.cuh"
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

// The PML coefficient tables (PlainTabs): block y = component, block z =
// table pair; the expressions are plain_component's, so every value is the
// one the per-cell code computes at that coordinate.
struct PlainTabOut
{
  double *t[3][6];
};

__global__ void plain_tables_kernel (PlainHalf p, PlainTabOut o)
{
  const int ci = blockIdx.y, role = blockIdx.z;
  const CompDev &c = p.comp[ci];
  if (!c.exists)
    return;
  const double *const *sig = p.dmp ? p.sigc[ci] : p.sigma;
  const int axis = role == 0 ? c.sig_cacb : (role == 1 ? c.sig5 : c.sig4);
  const int n = p.g.n[axis];
  const double eps0 = kEps0Dev;
  const double dt = p.g.dt;
  const double dx = p.g.dx;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x)
  {
    bool inside = true;
    for (int j = 0; j < c.nmat; ++j)
      inside = inside && q + c.m[j][axis] >= 0 && q + c.m[j][axis] < n;
    if (!inside)
      continue;
    const double material = sigma_avg (c, sig[axis], axis, q, q, q);
    if (role == 0)
    {
      double dd = (2 * eps0 * 1.0 + material * dt);
      o.t[ci][0][q] = (2 * eps0 * 1.0 - material * dt) / dd;
      o.t[ci][1][q] = (2 * eps0 * dt / dx) / dd;
    }
    else if (role == 1)
    {
      double dd5 = (2 * eps0 * 1.0 + material * dt);
      o.t[ci][2][q] = (2 * eps0 * 1.0 - material * dt) / dd5;
      o.t[ci][3][q] = dd5;
    }
    else
    {
      o.t[ci][4][q] = (2 * eps0 * 1.0 + material * dt);
      o.t[ci][5][q] = (2 * eps0 * 1.0 - material * dt);
    }
  }
}

// One component of one half-step over every interior cell (the arithmetic
// of plain_component, parameters resolved before the cell loop).
template <bool PML, bool META, bool TFSF>
__global__ void __launch_bounds__ (256) plain_fast_kernel (const __grid_constant__ PlainHalf p,
                                                           const __grid_constant__ PlainTabs tb, int ncomp,
                                                           int inc_len, int *err)
{
  // block b updates component b % ncomp (of the existing ones) on cell block
  // b / ncomp: the blocks that read the same opposite-family cells run
  // together, so the later ones find them in L2
  int ci = 0;
  for (int k = 0, left = (int) (blockIdx.x % ncomp); k < 3; ++k)
    if (p.comp[k].exists && left-- == 0)
    {
      ci = k;
      break;
    }
  const int64_t cblock = blockIdx.x / ncomp, cgrid = gridDim.x / ncomp;
  const GeomDev &g = p.g;
  const CompDev &c = p.comp[ci];
  const int64_t sx = (int64_t) g.n[1] * g.n[2], sy = g.n[2];
  const int64_t d11 = c.d11[0] * sx + c.d11[1] * sy + c.d11[2];
  const int64_t d12 = c.d12[0] * sx + c.d12[1] * sy + c.d12[2];
  const int64_t d21 = c.d21[0] * sx + c.d21[1] * sy + c.d21[2];
  const int64_t d22 = c.d22[0] * sx + c.d22[1] * sy + c.d22[2];
  const int nmat = c.nmat;
  int64_t mo[4];
#pragma unroll
  for (int j = 0; j < 4; ++j)
    mo[j] = c.m[j][0] * sx + c.m[j][1] * sy + c.m[j][2];
  const double *o1 = p.opp[c.opp1];
  const double *o2 = p.opp[c.opp2];
  const double *mat = p.dmp ? p.matc[ci] : p.mat;
  double *g0 = PML ? p.dd[ci][0] : p.f[ci][0];
  const double *g1 = PML ? p.dd[ci][1] : p.f[ci][1];
  const int ax_c = c.sig_cacb, ax5 = c.sig5, ax4 = c.sig4;
  const double *t_ca = tb.t[ci][0], *t_cb = tb.t[ci][1], *t_ca2 = tb.t[ci][2], *t_dd5 = tb.t[ci][3];
  const double *t_n4p = tb.t[ci][4], *t_n4m = tb.t[ci][5];
  const double dt = g.dt, dx = g.dx, mm = p.mat_modifier;
  double *f0 = p.f[ci][0];
  const double *f1 = p.f[ci][1];
  auto avg = [&] (const double *m, int64_t id) -> double {
    const double v0 = m[id + mo[0]];
    const double v1 = nmat > 1 ? m[id + mo[1]] : 0.0;
    const double v2 = nmat > 2 ? m[id + mo[2]] : 0.0;
    const double v3 = nmat > 3 ? m[id + mo[3]] : 0.0;
    return avg_points (nmat, v0, v1, v2, v3);
  };

  const int ix = (g.drop & 1) ? 1 : g.n[0] - 2;
  const int iy = (g.drop & 2) ? 1 : g.n[1] - 2;
  const int iz = (g.drop & 4) ? 1 : g.n[2] - 2;
  const int oz = (g.drop & 4) ? 0 : 1, oy = (g.drop & 2) ? 0 : 1, ox = (g.drop & 1) ? 0 : 1;
  for (CellWalk w (cblock * blockDim.x + threadIdx.x, cgrid * blockDim.x, ix, iy, iz); w.ok (); w.next ())
  {
    const int z = w.cz + oz, y = w.cy + oy, x = w.cx + ox;
    const int64_t id = x * sx + y * sy + z;
    const int pos[3] = {x, y, z};
    double val = g1[id];
    double ca, cb;
    if (PML)
    {
      const int q = ax_c == 0 ? x : (ax_c == 1 ? y : z);
      ca = t_ca[q];
      cb = t_cb[q];
    }
    else
    {
      double material = avg (mat, id);
      ca = 1.0;
      cb = dt / (material * mm * dx);
    }
    double v0 = 0.0, v1 = 0.0, v2 = 0.0, v3 = 0.0;
    if (o1)
    {
      v0 = o1[id + d11];
      v1 = o1[id + d12];
    }
    if (o2)
    {
      v2 = o2[id + d21];
      v3 = o2[id + d22];
    }
    if (TFSF)
    {
      for (int t = 0; t < c.nterms; ++t)
      {
        const TermDev &tm = c.term[t];
        if (x >= tm.lo[0] && x < tm.hi[0] && y >= tm.lo[1] && y < tm.hi[1] && z >= tm.lo[2] && z < tm.hi[2])
        {
          double diff = incident_value (g, p.inc, inc_len, err, tm.inc_comp, x + tm.aux[0], y + tm.aux[1],
                                        z + tm.aux[2]);
          if (tm.negate < 0)
            diff *= -1.0;
          if (tm.slot == 0)
            v0 -= diff;
          else if (tm.slot == 1)
            v1 -= diff;
          else if (tm.slot == 2)
            v2 -= diff;
          else
            v3 -= diff;
        }
      }
    }
    double tmp = v1 - v0 - v3 + v2 - 0.0 * dx;
    double nv = val * ca + tmp * cb;
    g0[id] = nv;
    if (!PML)
      continue;
    if (META)
    {
      double cur = p.dd[ci][0][id], prev = p.dd[ci][1][id], pprev = p.dd[ci][2][id];
      double prev1 = p.d1[ci][1][id], pprev1 = p.d1[ci][2][id];
      double material = avg (mat, id);
      const double *om = p.omega, *ga = p.gamma;
      double omega, gamma;
      if (nmat == 2)
      {
        omega = (om[id + mo[0]] + om[id + mo[1]]) / 2.0;
        gamma = (ga[id + mo[0]] + ga[id + mo[1]]) / 2.0;
      }
      else
      {
        omega = (om[id + mo[0]] + om[id + mo[1]] + om[id + mo[2]] + om[id + mo[3]]) / 4.0;
        gamma = (ga[id + mo[0]] + ga[id + mo[1]] + ga[id + mo[2]] + ga[id + mo[3]]) / 4.0;
      }
      double sq = dt * omega;
      double A = 4 * mm * material + 2 * dt * mm * material * gamma + mm * (sq * sq);
      double b0 = (4 + 2 * dt * gamma) / A;
      double b1 = -8 / A;
      double b2 = (4 - 2 * dt * gamma) / A;
      double a1 = (2 * mm * (sq * sq) - 8 * mm * material) / A;
      double a2 = (4 * mm * material - 2 * dt * mm * material * gamma + mm * (sq * sq)) / A;
      p.d1[ci][0][id] = cur * b0 + prev * b1 + pprev * b2 - prev1 * a1 - pprev1 * a2;
    }
    double prev_eh = f1[id];
    double *const *src = META ? p.d1[ci] : p.dd[ci];
    double cur_db = src[0][id];
    double prev_db = src[1][id];
    double material1 = avg (mat, id);
    double modifier = material1 * mm;
    if (META)
      modifier = 1;
    const int q5 = pos[ax5], q4 = pos[ax4];
    double dd5 = t_dd5[q5];
    double ca2 = t_ca2[q5];
    double cb2 = (t_n4p[q4] / (modifier)) / dd5;
    double cc2 = (t_n4m[q4] / (modifier)) / dd5;
    f0[id] = prev_eh * ca2 + cur_db * cb2 - prev_db * cc2;
  }
}

int launch_plain_tables (const PlainHalf &p, double *const out[3][6], cudaStream_t s)
{
  PlainTabOut o;
  for (int ci = 0; ci < 3; ++ci)
    for (int j = 0; j < 6; ++j)
      o.t[ci][j] = out[ci][j];
  plain_tables_kernel<<<dim3 (4, 3, 3), 256, 0, s>>> (p, o);
  return 1;
}

int launch_plain_fast (const PlainHalf &p, const PlainTabs &t, int inc_len, int *err, int sm_count,
                       cudaStream_t s)
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
  int ncomp = 0;
  for (int ci = 0; ci < 3; ++ci)
    ncomp += p.comp[ci].exists ? 1 : 0;
  if (ncomp == 0)
    return 0;
  auto kern = p.use_pml ? (p.use_meta ? (p.use_tfsf ? plain_fast_kernel<true, true, true>
                                                    : plain_fast_kernel<true, true, false>)
                                      : (p.use_tfsf ? plain_fast_kernel<true, false, true>
                                                    : plain_fast_kernel<true, false, false>))
                        : (p.use_tfsf ? plain_fast_kernel<false, false, true> : plain_fast_kernel<false, false, false>);
  kern<<<(unsigned) (blocks * ncomp), 256, 0, s>>> (p, t, ncomp, inc_len, err);
  return 1;
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
