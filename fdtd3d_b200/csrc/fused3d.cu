// fused3d.cu - one-sweep E+H leapfrog step for the 3-D FP32 / FP16-storage
// forms (uniform mu).
//
// Per time step every field value is read once from the "old" buffers and
// written once to the "new" buffers (E, H and the PML auxiliaries are double
// buffered).  Because nothing read is ever written in the same sweep, tiles
// need no inter-CTA synchronisation: each CTA owns a (y, z) tile and an x
// chunk, marches x, and recomputes from old data the few E values it needs
// on the high-side ring of its tile and on the plane after its chunk.
//
// Per x-plane a CTA of (TZ+1) x (TY+1) threads:
//   1. stages H_old(x) (+ low-side halo) and eps(x) (+ high-side ring) in
//      shared memory; E_old(x) and H_old(x-1) stay in registers;
//   2. computes E_new(x) on the tile plus its ring (curl, TF/SF, PML, point
//      source) - the ring values are only used, never stored;
//   3. computes H_new(x-1) on the tile from E_new(x-1) (shared memory, kept
//      from the previous plane) and E_new(x) (registers);
//   4. stores E_new(x) and H_new(x-1) for the owned cells.
// The arithmetic is the formulation of fast_kernels.cu (H stored as
// eta0*H, PML auxiliaries D/eps0 and c*B touched only in PML cells).
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "fused3d.h"

namespace fdtdb {

namespace {

template <typename T>
__device__ __forceinline__ float ldf (const T *p, size_t i);
template <>
__device__ __forceinline__ float ldf<float> (const float *p, size_t i)
{
  return __ldg (p + i);
}
template <>
__device__ __forceinline__ float ldf<__half> (const __half *p, size_t i)
{
  return __half2float (__ldg (p + i));
}

template <typename T>
__device__ __forceinline__ void stf (T *p, size_t i, float v);
template <>
__device__ __forceinline__ void stf<float> (float *p, size_t i, float v)
{
  p[i] = v;
}
template <>
__device__ __forceinline__ void stf<__half> (__half *p, size_t i, float v)
{
  p[i] = __float2half_rn (v);
}

__device__ __forceinline__ double inc_at (const GeomDev &g, const double *inc, int inc_len, int *err, int k,
                                          int px, int py, int pz)
{
  double d_diff = k >= 3 ? 0.5 : 0.0;
  double x = ((double) px + g.min_fp[k][0]) - g.zero_inc[0];
  double y = ((double) py + g.min_fp[k][1]) - g.zero_inc[1];
  double z = ((double) pz + g.min_fp[k][2]) - g.zero_inc[2];
  double d = x * g.s1 * g.c2 + y * g.s1 * g.s2 + z * g.c1 - d_diff;
  int i1 = (int) d;
  double pr2 = d - (double) i1;
  if (i1 < 0 || i1 + 1 >= inc_len)
  {
    *err = 1;
    return 0.0;
  }
  return (inc[i1] * (1 - pr2) + inc[i1 + 1] * pr2) * g.proj[k];
}

// TF/SF corrections of component k at (x, y, z): subtract the incident
// projection from the neighbour slot each matching term names.
__device__ __forceinline__ void tfsf_apply (const FusedParams &p, int k, const double *inc, int *err, int x, int y,
                                            int z, float &v0, float &v1, float &v2, float &v3)
{
  const CompDev &c = p.comp[k];
  for (int t = 0; t < c.nterms; ++t)
  {
    const TermDev &tm = c.term[t];
    if (x >= tm.lo[0] && x < tm.hi[0] && y >= tm.lo[1] && y < tm.hi[1] && z >= tm.lo[2] && z < tm.hi[2])
    {
      double diff = inc_at (p.g, inc, p.inc_len, err, tm.inc_comp, x + tm.aux[0], y + tm.aux[1], z + tm.aux[2]);
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

// Update of one component at one cell given its curl: interior or PML.
// `store_aux` is false for recomputed ring values (owned by another tile).
__device__ __forceinline__ float update (const FusedParams &p, int k, bool interior, float f, float curl, float inv_m,
                                         int x, int y, int z, size_t id, bool store_aux)
{
  if (interior)
    return f + p.courant * inv_m * curl;
  const int pos[3] = {x, y, z};
  const CompDev &c = p.comp[k];
  const float ca1 = p.tab[k][0][pos[c.sig_cacb]];
  const float sq1 = p.tab[k][1][pos[c.sig_cacb]];
  const float p5 = p.tab[k][2][pos[c.sig5]];
  const float q5 = p.tab[k][3][pos[c.sig5]];
  const float g4p = p.tab[k][4][pos[c.sig4]];
  const float g4m = p.tab[k][5][pos[c.sig4]];
  const float xo = p.aux_old[k][id];
  const float xn = ca1 * xo + sq1 * curl;
  if (store_aux)
    p.aux_new[k][id] = xn;
  return p5 * f + (g4p * xn - g4m * xo) * q5 * inv_m;
}

// Is coordinate v one of the (up to 4) TF/SF face planes of an axis?
__device__ __forceinline__ bool on_face (const int *planes, int v)
{
  return v == planes[0] || v == planes[1] || v == planes[2] || v == planes[3];
}

template <typename T, int TY, int TZ>
__global__ void __launch_bounds__ ((TY + 1) * (TZ + 1)) fused3d_kernel (FusedParams p, int *err)
{
  const int nx = p.g.n[0], ny = p.g.n[1], nz = p.g.n[2];
  const int tz = threadIdx.x;
  const int ty = threadIdx.y;
  const int y0 = 1 + blockIdx.y * TY;
  const int z0 = 1 + blockIdx.x * TZ;
  const int y = y0 + ty;
  const int z = z0 + tz;
  const int xa = 1 + blockIdx.z * p.x_chunk;
  const int xb = min (xa + p.x_chunk - 1, nx - 2);
  const bool valid = y <= ny - 1 && z <= nz - 1;
  const bool inner = y <= ny - 2 && z <= nz - 2;          // y, z >= 1 always
  const bool owner = tz < TZ && ty < TY && inner;
  const size_t sx = (size_t) ny * nz;
  const size_t col = (size_t) y * nz + z;

  __shared__ float sH[3][TY + 2][TZ + 2];
  __shared__ float sE[3][TY + 1][TZ + 1];
  __shared__ float sEps[TY + 2][TZ + 2];

  // PML classification: y, z are fixed per thread, x is uniform per plane
  bool yz_in[6];
#pragma unroll
  for (int k = 0; k < 6; ++k)
    yz_in[k] = !p.use_pml || (y >= p.ilo[k][1] && y < p.ihi[k][1] && z >= p.ilo[k][2] && z < p.ihi[k][2]);
  const bool yz_face = p.use_tfsf && (on_face (p.face[1], y) || on_face (p.face[2], z));

  const T *Eo[3] = {(const T *) p.e_old[0], (const T *) p.e_old[1], (const T *) p.e_old[2]};
  const T *Ho[3] = {(const T *) p.h_old[0], (const T *) p.h_old[1], (const T *) p.h_old[2]};
  T *En[3] = {(T *) p.e_new[0], (T *) p.e_new[1], (T *) p.e_new[2]};
  T *Hn[3] = {(T *) p.h_new[0], (T *) p.h_new[1], (T *) p.h_new[2]};

  // state at x = xa - 1: H_old and E_new (= recomputed below only for x >= xa;
  // the plane before the chunk is only needed by H_new(xa - 1), not owned)
  float hp[3] = {0.f, 0.f, 0.f};
  float ep[3] = {0.f, 0.f, 0.f};
  if (valid)
  {
    size_t id = (size_t) (xa - 1) * sx + col;
#pragma unroll
    for (int c = 0; c < 3; ++c)
      hp[c] = ldf (Ho[c], id);
  }

  for (int x = xa; x <= xb + 1; ++x)
  {
    const size_t id = (size_t) x * sx + col;
    const bool xin = x <= nx - 2;
    // 1. stage
    float eo[3] = {0.f, 0.f, 0.f};
    float epsx1 = 1.f;
    if (valid)
    {
#pragma unroll
      for (int c = 0; c < 3; ++c)
      {
        sH[c][ty + 1][tz + 1] = ldf (Ho[c], id);
        eo[c] = ldf (Eo[c], id);
      }
      if (p.eps)
      {
        sEps[ty][tz] = __ldg (p.eps + id);
        if (x + 1 <= nx - 1)
          epsx1 = __ldg (p.eps + id + sx);
      }
    }
    else
    {
#pragma unroll
      for (int c = 0; c < 3; ++c)
        sH[c][ty + 1][tz + 1] = 0.f;
      sEps[ty][tz] = 1.f;
    }
    if (ty == 0)
    {
      bool v = z <= nz - 1;
      size_t hid = id - nz;
      sH[0][0][tz + 1] = v ? ldf (Ho[0], hid) : 0.f;
      sH[2][0][tz + 1] = v ? ldf (Ho[2], hid) : 0.f;
    }
    if (tz == 0)
    {
      bool v = y <= ny - 1;
      size_t hid = id - 1;
      sH[0][ty + 1][0] = v ? ldf (Ho[0], hid) : 0.f;
      sH[1][ty + 1][0] = v ? ldf (Ho[1], hid) : 0.f;
    }
    if (p.eps)
    {
      if (ty == TY)
        sEps[TY + 1][tz] = (y + 1 <= ny - 1 && z <= nz - 1) ? __ldg (p.eps + id + nz) : 1.f;
      if (tz == TZ)
        sEps[ty][TZ + 1] = (z + 1 <= nz - 1 && y <= ny - 1) ? __ldg (p.eps + id + 1) : 1.f;
    }
    __syncthreads ();

    // 2. E_new(x) on tile + ring
    float en[3] = {eo[0], eo[1], eo[2]};
    if (inner && xin)
    {
      float inv[3] = {1.f, 1.f, 1.f};
      if (p.eps)
      {
        const float e0 = sEps[ty][tz];
        inv[0] = __fdividef (2.f, e0 + epsx1);
        inv[1] = __fdividef (2.f, e0 + sEps[ty + 1][tz]);
        inv[2] = __fdividef (2.f, e0 + sEps[ty][tz + 1]);
      }
      // Ex: Hz(y-1), Hz, Hy(z-1), Hy
      float a0 = sH[2][ty][tz + 1], a1 = sH[2][ty + 1][tz + 1], a2 = sH[1][ty + 1][tz], a3 = sH[1][ty + 1][tz + 1];
      // Ey: Hx(z-1), Hx, Hz(x-1), Hz
      float b0 = sH[0][ty + 1][tz], b1 = sH[0][ty + 1][tz + 1], b2 = hp[2], b3 = sH[2][ty + 1][tz + 1];
      // Ez: Hy(x-1), Hy, Hx(y-1), Hx
      float c0 = hp[1], c1 = sH[1][ty + 1][tz + 1], c2 = sH[0][ty][tz + 1], c3 = sH[0][ty + 1][tz + 1];
      if (yz_face || (p.use_tfsf && on_face (p.face[0], x)))
      {
        tfsf_apply (p, 0, p.inc_h, err, x, y, z, a0, a1, a2, a3);
        tfsf_apply (p, 1, p.inc_h, err, x, y, z, b0, b1, b2, b3);
        tfsf_apply (p, 2, p.inc_h, err, x, y, z, c0, c1, c2, c3);
      }
      const bool st_aux = owner && x <= xb;
      en[0] = update (p, 0, yz_in[0] && x >= p.ilo[0][0] && x < p.ihi[0][0], eo[0], (a1 - a0) - (a3 - a2), inv[0],
                      x, y, z, id, st_aux);
      en[1] = update (p, 1, yz_in[1] && x >= p.ilo[1][0] && x < p.ihi[1][0], eo[1], (b1 - b0) - (b3 - b2), inv[1],
                      x, y, z, id, st_aux);
      en[2] = update (p, 2, yz_in[2] && x >= p.ilo[2][0] && x < p.ihi[2][0], eo[2], (c1 - c0) - (c3 - c2), inv[2],
                      x, y, z, id, st_aux);
      if (p.ps_mask & 7)
      {
        if (x == p.ps[0] && y == p.ps[1] && z == p.ps[2])
        {
          float v = (float) p.src[p.src_index];
#pragma unroll
          for (int c = 0; c < 3; ++c)
            if (p.ps_mask & (1 << c))
              en[c] = v;
        }
      }
      if (owner && x <= xb)
      {
#pragma unroll
        for (int c = 0; c < 3; ++c)
          stf (En[c], id, en[c]);
      }
    }

    // 3. H_new(x-1) on the tile
    const int xh = x - 1;
    if (owner && xh >= xa)
    {
      const size_t hid = id - sx;
      // Hx: Ey, Ey(z+1), Ez, Ez(y+1)
      float a0 = ep[1], a1 = sE[1][ty][tz + 1], a2 = ep[2], a3 = sE[2][ty + 1][tz];
      // Hy: Ez, Ez(x+1), Ex, Ex(z+1)
      float b0 = ep[2], b1 = en[2], b2 = ep[0], b3 = sE[0][ty][tz + 1];
      // Hz: Ex, Ex(y+1), Ey, Ey(x+1)
      float c0 = ep[0], c1 = sE[0][ty + 1][tz], c2 = ep[1], c3 = en[1];
      if (yz_face || (p.use_tfsf && on_face (p.face[0], xh)))
      {
        tfsf_apply (p, 3, p.inc_e, err, xh, y, z, a0, a1, a2, a3);
        tfsf_apply (p, 4, p.inc_e, err, xh, y, z, b0, b1, b2, b3);
        tfsf_apply (p, 5, p.inc_e, err, xh, y, z, c0, c1, c2, c3);
      }
      float hn[3];
      hn[0] = update (p, 3, yz_in[3] && xh >= p.ilo[3][0] && xh < p.ihi[3][0], hp[0], (a1 - a0) - (a3 - a2), 1.f,
                      xh, y, z, hid, true);
      hn[1] = update (p, 4, yz_in[4] && xh >= p.ilo[4][0] && xh < p.ihi[4][0], hp[1], (b1 - b0) - (b3 - b2), 1.f,
                      xh, y, z, hid, true);
      hn[2] = update (p, 5, yz_in[5] && xh >= p.ilo[5][0] && xh < p.ihi[5][0], hp[2], (c1 - c0) - (c3 - c2), 1.f,
                      xh, y, z, hid, true);
      if (p.ps_mask & 56)
      {
        if (xh == p.ps[0] && y == p.ps[1] && z == p.ps[2])
        {
          float v = (float) p.src[p.src_index + 1] * p.ps_scale_h;
#pragma unroll
          for (int c = 0; c < 3; ++c)
            if (p.ps_mask & (8 << c))
              hn[c] = v;
        }
      }
#pragma unroll
      for (int c = 0; c < 3; ++c)
        stf (Hn[c], hid, hn[c]);
    }
    __syncthreads ();

    // 4. carry plane x into the next iteration
#pragma unroll
    for (int c = 0; c < 3; ++c)
    {
      sE[c][ty][tz] = valid ? en[c] : 0.f;
      ep[c] = en[c];
      hp[c] = sH[c][ty + 1][tz + 1];
    }
  }
}

}  // namespace

int launch_fused3d (const FusedParams &p, int *err, cudaStream_t s)
{
  constexpr int TY = 8, TZ = 32;
  const int ny = p.g.n[1], nz = p.g.n[2], nx = p.g.n[0];
  dim3 block (TZ + 1, TY + 1);
  dim3 grid ((nz - 2 + TZ - 1) / TZ, (ny - 2 + TY - 1) / TY, (nx - 2 + p.x_chunk - 1) / p.x_chunk);
  if (p.fp16)
    fused3d_kernel<__half, TY, TZ><<<grid, block, 0, s>>> (p, err);
  else
    fused3d_kernel<float, TY, TZ><<<grid, block, 0, s>>> (p, err);
  return 1;
}

}  // namespace fdtdb
