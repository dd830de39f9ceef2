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
#include <climits>
#include <algorithm>
#include <cuda_runtime.h>

#include "fused3d.h"
#include "incident_dev.cuh"

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

// Drude coefficients of component k at (x, y, z) in the scaled formulation
// (X = D/eps0 or c*B, Z = D1 or eta0*B1): the reference's b0..a2
// (Source/Scheme/InternalScheme.inc.h:2527-2532) multiplied through by the
// vacuum constant, with the plasma frequency and collision rate averaged as
// getMetaMaterial does (two points for E, the plain mean of four for H).
__device__ __forceinline__ void drude_coeffs (const FusedParams &p, int k, int x, int y, int z, float c[5])
{
  const int ny = p.g.n[1], nz = p.g.n[2];
  const size_t stride[3] = {(size_t) ny * nz, (size_t) nz, 1};
  const size_t id = ((size_t) x * ny + y) * nz + z;
  const int side = k >= 3 ? 1 : 0;
  const float *om = p.omega[side];
  const float *ga = p.gamma[side];
  float w, g, m = 1.f;
  if (k < 3)
  {
    const size_t j = id + stride[k];
    w = 0.5f * (om[id] + om[j]);
    g = 0.5f * (ga[id] + ga[j]);
    if (p.eps)
      m = 0.5f * (p.eps[id] + p.eps[j]);
  }
  else
  {
    const int a = k - 3;
    const int lo = a == 0 ? 1 : 0;
    const int hi = a == 2 ? 1 : 2;
    const size_t j1 = id + stride[hi], j2 = id + stride[lo], j3 = id + stride[lo] + stride[hi];
    w = 0.25f * (om[id] + om[j1] + om[j2] + om[j3]);
    g = 0.25f * (ga[id] + ga[j1] + ga[j2] + ga[j3]);
  }
  const float dt = p.dt;
  const float sq = (dt * w) * (dt * w);
  const float inv = 1.f / (4.f * m + 2.f * dt * m * g + sq);
  c[0] = (4.f + 2.f * dt * g) * inv;
  c[1] = -8.f * inv;
  c[2] = (4.f - 2.f * dt * g) * inv;
  c[3] = (2.f * sq - 8.f * m) * inv;
  c[4] = (4.f * m - 2.f * dt * m * g + sq) * inv;
}

// Dispersive cell: curl step of X (PML coefficients, sigma = 0 inside),
// Drude recurrence to Z, then F from Z with modifier 1 (the reference's
// metamaterial PML path, InternalScheme.inc.h:2551-2640).
__device__ __forceinline__ float update_drude (const FusedParams &p, int k, float f, float curl, int x, int y, int z,
                                               size_t id, bool store)
{
  const int pos[3] = {x, y, z};
  const CompDev &c = p.comp[k];
  const float ca1 = p.tab[k][0][pos[c.sig_cacb]];
  const float sq1 = p.tab[k][1][pos[c.sig_cacb]];
  const float p5 = p.tab[k][2][pos[c.sig5]];
  const float q5 = p.tab[k][3][pos[c.sig5]];
  const float g4p = p.tab[k][4][pos[c.sig4]];
  const float g4m = p.tab[k][5][pos[c.sig4]];
  const float xo = p.aux_old[k][id];
  const float xpp = p.xpp_old[k][id];
  const float zo = p.z_old[k][id];
  const float zpp = p.zpp_old[k][id];
  float b[5];
  drude_coeffs (p, k, x, y, z, b);
  const float xn = ca1 * xo + sq1 * curl;
  const float zn = b[0] * xn + b[1] * xo + b[2] * xpp - b[3] * zo - b[4] * zpp;
  if (store)
  {
    p.aux_new[k][id] = xn;
    p.xpp_new[k][id] = xo;
    p.z_new[k][id] = zn;
    p.zpp_new[k][id] = zo;
  }
  return p5 * f + (g4p * zn - g4m * zo) * q5;
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

// Per-component update with the component fixed at compile time, so the
// PML table axes are constants (axis a = K % 3; curl-step coefficients along
// a + 1, E-from-D coefficients along a + 2 and a, as the reference's
// SigmaY/SigmaZ/SigmaX choice for Ex and its rotations).
template <int K>
__device__ __forceinline__ float update_k (const FusedParams &p, bool interior, float f, float curl, float inv_m,
                                           int x, int y, int z, size_t id, bool store)
{
  if (interior)
    return f + p.courant * inv_m * curl;
  constexpr int A = K % 3, C1 = (K + 1) % 3, C2 = (K + 2) % 3;
  const int pos[3] = {x, y, z};
  const float ca1 = __ldg (p.tab[K][0] + pos[C1]);
  const float sq1 = __ldg (p.tab[K][1] + pos[C1]);
  const float p5 = __ldg (p.tab[K][2] + pos[C2]);
  const float q5 = __ldg (p.tab[K][3] + pos[C2]);
  const float g4p = __ldg (p.tab[K][4] + pos[A]);
  const float g4m = __ldg (p.tab[K][5] + pos[A]);
  const float xo = p.aux_old[K][id];
  const float xn = ca1 * xo + sq1 * curl;
  if (store)
    p.aux_new[K][id] = xn;
  return p5 * f + (g4p * xn - g4m * xo) * q5 * inv_m;
}

template <int K, bool META>
__device__ __forceinline__ float update_any (const FusedParams &p, unsigned fl, bool interior, float f, float curl,
                                             float inv_m, int x, int y, int z, size_t id, bool store)
{
  if (META && (fl & (1u << K)))
    return update_drude (p, K, f, curl, x, y, z, id, store);
  return update_k<K> (p, interior, f, curl, inv_m, x, y, z, id, store);
}

// One-sweep kernel.  CTA = W warps stacked along y; a warp covers 32 z
// positions (lanes 0..30 owned, lane 31 the z ring) and R consecutive y
// rows per thread, so each thread keeps a small column of cells in
// registers.  The last row of the last warp is the CTA's y ring, so a CTA
// owns 31 x (R*W - 1) cells of every x plane of its chunk.  Neighbours move
// by warp shuffles (z), registers (y inside a warp, x between planes) and
// a parity-double-buffered shared row per warp boundary (y), so one
// __syncthreads per plane is enough.
template <typename T, int R, int W, bool META>
__global__ void __launch_bounds__ (32 * W) fused3d_kernel (FusedParams p, int *err)
{
  const int nx = p.g.n[0], ny = p.g.n[1], nz = p.g.n[2];
  const int lane = threadIdx.x;
  const int w = threadIdx.y;
  const int z0 = 1 + blockIdx.x * 31;
  const int z = z0 + lane;
  const int yw = 1 + blockIdx.y * (R * W - 1) + w * R;
  const int xa = 1 + blockIdx.z * p.x_chunk;
  const int xb = min (xa + p.x_chunk - 1, nx - 2);
  const bool zvalid = z <= nz - 1;
  const bool zinner = z <= nz - 2;
  const bool zown = lane < 31 && zinner;
  const unsigned FULL = 0xffffffffu;
  const size_t sx = (size_t) ny * nz;

  __shared__ float sHb[2][W + 1][2][32];   // [parity][warp + 1][Hz, Hx][lane]: row above each warp
  __shared__ float sEb[2][W][2][32];       // [parity][warp][Ex, Ez][lane]: E_new of each warp's first row

  bool rvalid[R], rinner[R], rown[R];
  unsigned yzin = 0;                       // bit k*R + r: component k, row r has sigma == 0 along y and z
  unsigned face = 0;                       // bit r: row r lies on a TF/SF face plane along y or z
#pragma unroll
  for (int r = 0; r < R; ++r)
  {
    const int y = yw + r;
    rvalid[r] = y <= ny - 1 && zvalid;
    rinner[r] = y <= ny - 2 && zinner;
    rown[r] = rinner[r] && lane < 31 && !(w == W - 1 && r == R - 1);
#pragma unroll
    for (int k = 0; k < 6; ++k)
      if (!p.use_pml || (y >= p.ilo[k][1] && y < p.ihi[k][1] && z >= p.ilo[k][2] && z < p.ihi[k][2]))
        yzin |= 1u << (k * R + r);
    if (p.use_tfsf && (on_face (p.face[1], y) || on_face (p.face[2], z)))
      face |= 1u << r;
  }

  const T *Ho0 = (const T *) p.h_old[0], *Ho1 = (const T *) p.h_old[1], *Ho2 = (const T *) p.h_old[2];
  const T *Eo0 = (const T *) p.e_old[0], *Eo1 = (const T *) p.e_old[1], *Eo2 = (const T *) p.e_old[2];
  T *En0 = (T *) p.e_new[0], *En1 = (T *) p.e_new[1], *En2 = (T *) p.e_new[2];
  T *Hn0 = (T *) p.h_new[0], *Hn1 = (T *) p.h_new[1], *Hn2 = (T *) p.h_new[2];
  const float *eps = p.eps;

  float hp[3][R], ep[3][R], epsc[R];
  unsigned char flp[R];
  {
    const size_t b0 = (size_t) (xa - 1) * sx + (size_t) yw * nz + z;
#pragma unroll
    for (int r = 0; r < R; ++r)
    {
      const size_t id = b0 + (size_t) r * nz;
      hp[0][r] = rvalid[r] ? ldf (Ho0, id) : 0.f;
      hp[1][r] = rvalid[r] ? ldf (Ho1, id) : 0.f;
      hp[2][r] = rvalid[r] ? ldf (Ho2, id) : 0.f;
      ep[0][r] = ep[1][r] = ep[2][r] = 0.f;
      epsc[r] = (eps && rvalid[r]) ? __ldg (eps + id + sx) : 1.f;
      flp[r] = (META && rvalid[r]) ? p.dflag[id] : 0;
    }
  }

  for (int x = xa; x <= xb + 1; ++x)
  {
    const int par = x & 1;
    const size_t b = (size_t) x * sx + (size_t) yw * nz + z;
    // ---- loads of plane x (independent, all in flight together)
    float h[3][R], e[3][R], epsn[R];
    unsigned char fl[R];
#pragma unroll
    for (int r = 0; r < R; ++r)
    {
      const size_t id = b + (size_t) r * nz;
      h[0][r] = rvalid[r] ? ldf (Ho0, id) : 0.f;
      h[1][r] = rvalid[r] ? ldf (Ho1, id) : 0.f;
      h[2][r] = rvalid[r] ? ldf (Ho2, id) : 0.f;
      e[0][r] = rvalid[r] ? ldf (Eo0, id) : 0.f;
      e[1][r] = rvalid[r] ? ldf (Eo1, id) : 0.f;
      e[2][r] = rvalid[r] ? ldf (Eo2, id) : 0.f;
      epsn[r] = (eps && rvalid[r] && x + 1 <= nx - 1) ? __ldg (eps + id + sx) : 1.f;
      fl[r] = (META && rvalid[r]) ? p.dflag[id] : 0;
    }
    float hzl_x[R], hzl_y[R], epz[R];
#pragma unroll
    for (int r = 0; r < R; ++r)
    {
      const size_t id = b + (size_t) r * nz;
      const bool rv = yw + r <= ny - 1;
      hzl_x[r] = (lane == 0 && rv) ? ldf (Ho0, id - 1) : 0.f;
      hzl_y[r] = (lane == 0 && rv) ? ldf (Ho1, id - 1) : 0.f;
      epz[r] = (eps && lane == 31 && rv && z + 1 <= nz - 1) ? __ldg (eps + id + 1) : 1.f;
    }
    const float epsy = (eps && zvalid && yw + R <= ny - 1) ? __ldg (eps + b + (size_t) R * nz) : 1.f;
    if (w == 0)
    {
      sHb[par][0][0][lane] = zvalid ? ldf (Ho2, b - nz) : 0.f;
      sHb[par][0][1][lane] = zvalid ? ldf (Ho0, b - nz) : 0.f;
    }
    sHb[par][w + 1][0][lane] = h[2][R - 1];
    sHb[par][w + 1][1][lane] = h[0][R - 1];
    __syncthreads ();

    // ---- E_new(x), all rows of this warp including the rings
    const bool xin = x <= nx - 2;
    const bool xface = p.use_tfsf && on_face (p.face[0], x);
    const bool xi0 = x >= p.ilo[0][0] && x < p.ihi[0][0];
    const bool xi1 = x >= p.ilo[1][0] && x < p.ihi[1][0];
    const bool xi2 = x >= p.ilo[2][0] && x < p.ihi[2][0];
    const bool ps_e = (p.ps_mask & 7) && x == p.ps[0];
#pragma unroll
    for (int r = 0; r < R; ++r)
    {
      const float hz_ym = r == 0 ? sHb[par][w][0][lane] : h[2][r - 1];
      const float hx_ym = r == 0 ? sHb[par][w][1][lane] : h[0][r - 1];
      float hy_zm = __shfl_up_sync (FULL, h[1][r], 1);
      float hx_zm = __shfl_up_sync (FULL, h[0][r], 1);
      if (lane == 0)
      {
        hy_zm = hzl_y[r];
        hx_zm = hzl_x[r];
      }
      float ez1 = __shfl_down_sync (FULL, epsc[r], 1);
      if (lane == 31)
        ez1 = epz[r];
      if (rinner[r] && xin)
      {
        const int y = yw + r;
        const size_t id = b + (size_t) r * nz;
        float i0 = 1.f, i1 = 1.f, i2 = 1.f;
        if (eps)
        {
          const float e0 = epsc[r];
          i0 = __fdividef (2.f, e0 + epsn[r]);
          i1 = __fdividef (2.f, e0 + (r < R - 1 ? epsc[r + 1] : epsy));
          i2 = __fdividef (2.f, e0 + ez1);
        }
        float a0 = hz_ym, a1 = h[2][r], a2 = hy_zm, a3 = h[1][r];
        float b0 = hx_zm, b1 = h[0][r], b2 = hp[2][r], b3 = h[2][r];
        float c0 = hp[1][r], c1 = h[1][r], c2 = hx_ym, c3 = h[0][r];
        if (xface || (face & (1u << r)))
        {
          tfsf_apply (p, 0, p.inc_h, err, x, y, z, a0, a1, a2, a3);
          tfsf_apply (p, 1, p.inc_h, err, x, y, z, b0, b1, b2, b3);
          tfsf_apply (p, 2, p.inc_h, err, x, y, z, c0, c1, c2, c3);
        }
        const bool st = rown[r] && x <= xb;
        e[0][r] = update_any<0, META> (p, fl[r], xi0 && (yzin & (1u << (0 * R + r))), e[0][r],
                                       (a1 - a0) - (a3 - a2), i0, x, y, z, id, st);
        e[1][r] = update_any<1, META> (p, fl[r], xi1 && (yzin & (1u << (1 * R + r))), e[1][r],
                                       (b1 - b0) - (b3 - b2), i1, x, y, z, id, st);
        e[2][r] = update_any<2, META> (p, fl[r], xi2 && (yzin & (1u << (2 * R + r))), e[2][r],
                                       (c1 - c0) - (c3 - c2), i2, x, y, z, id, st);
        if (ps_e && y == p.ps[1] && z == p.ps[2])
        {
          const float v = (float) p.src[p.src_index];
          if (p.ps_mask & 1)
            e[0][r] = v;
          if (p.ps_mask & 2)
            e[1][r] = v;
          if (p.ps_mask & 4)
            e[2][r] = v;
        }
        if (st)
        {
          stf (En0, id, e[0][r]);
          stf (En1, id, e[1][r]);
          stf (En2, id, e[2][r]);
        }
      }
    }
    sEb[par][w][0][lane] = e[0][0];
    sEb[par][w][1][lane] = e[2][0];

    // ---- H_new(x - 1) on the owned rows
    const int xh = x - 1;
    if (xh >= xa)
    {
      const bool hface = p.use_tfsf && on_face (p.face[0], xh);
      const bool xi3 = xh >= p.ilo[3][0] && xh < p.ihi[3][0];
      const bool xi4 = xh >= p.ilo[4][0] && xh < p.ihi[4][0];
      const bool xi5 = xh >= p.ilo[5][0] && xh < p.ihi[5][0];
      const bool ps_h = (p.ps_mask & 56) && xh == p.ps[0];
#pragma unroll
      for (int r = 0; r < R; ++r)
      {
        const float ey_zp = __shfl_down_sync (FULL, ep[1][r], 1);
        const float ex_zp = __shfl_down_sync (FULL, ep[0][r], 1);
        if (rown[r])
        {
          const int y = yw + r;
          const size_t hid = b - sx + (size_t) r * nz;
          const float ez_yp = r < R - 1 ? ep[2][r + 1] : sEb[par ^ 1][w + 1 < W ? w + 1 : w][1][lane];
          const float ex_yp = r < R - 1 ? ep[0][r + 1] : sEb[par ^ 1][w + 1 < W ? w + 1 : w][0][lane];
          float a0 = ep[1][r], a1 = ey_zp, a2 = ep[2][r], a3 = ez_yp;
          float b0 = ep[2][r], b1 = e[2][r], b2 = ep[0][r], b3 = ex_zp;
          float c0 = ep[0][r], c1 = ex_yp, c2 = ep[1][r], c3 = e[1][r];
          if (hface || (face & (1u << r)))
          {
            tfsf_apply (p, 3, p.inc_e, err, xh, y, z, a0, a1, a2, a3);
            tfsf_apply (p, 4, p.inc_e, err, xh, y, z, b0, b1, b2, b3);
            tfsf_apply (p, 5, p.inc_e, err, xh, y, z, c0, c1, c2, c3);
          }
          float hn0 = update_any<3, META> (p, flp[r], xi3 && (yzin & (1u << (3 * R + r))), hp[0][r],
                                           (a1 - a0) - (a3 - a2), 1.f, xh, y, z, hid, true);
          float hn1 = update_any<4, META> (p, flp[r], xi4 && (yzin & (1u << (4 * R + r))), hp[1][r],
                                           (b1 - b0) - (b3 - b2), 1.f, xh, y, z, hid, true);
          float hn2 = update_any<5, META> (p, flp[r], xi5 && (yzin & (1u << (5 * R + r))), hp[2][r],
                                           (c1 - c0) - (c3 - c2), 1.f, xh, y, z, hid, true);
          if (ps_h && y == p.ps[1] && z == p.ps[2])
          {
            const float v = (float) p.src[p.src_index + 1] * p.ps_scale_h;
            if (p.ps_mask & 8)
              hn0 = v;
            if (p.ps_mask & 16)
              hn1 = v;
            if (p.ps_mask & 32)
              hn2 = v;
          }
          stf (Hn0, hid, hn0);
          stf (Hn1, hid, hn1);
          stf (Hn2, hid, hn2);
        }
      }
    }

    // ---- carry plane x
#pragma unroll
    for (int r = 0; r < R; ++r)
    {
      hp[0][r] = h[0][r];
      hp[1][r] = h[1][r];
      hp[2][r] = h[2][r];
      ep[0][r] = e[0][r];
      ep[1][r] = e[1][r];
      ep[2][r] = e[2][r];
      epsc[r] = epsn[r];
      flp[r] = fl[r];
    }
  }
}

// bit k of flags[cell]: component k averages a non-zero plasma frequency or
// collision rate (the averaging stencils of getMetaMaterial)
__global__ void drude_flags_kernel (unsigned char *flags, const float *ome, const float *gae, const float *omm,
                                    const float *gam, int nx, int ny, int nz)
{
  const size_t n = (size_t) nx * ny * nz;
  const size_t stride[3] = {(size_t) ny * nz, (size_t) nz, 1};
  for (size_t id = (size_t) blockIdx.x * blockDim.x + threadIdx.x; id < n; id += (size_t) gridDim.x * blockDim.x)
  {
    const int z = (int) (id % nz);
    const int y = (int) ((id / nz) % ny);
    const int x = (int) (id / stride[0]);
    const int pos[3] = {x, y, z};
    const int lim[3] = {nx, ny, nz};
    unsigned f = 0;
    for (int k = 0; k < 6; ++k)
    {
      const float *om = k < 3 ? ome : omm;
      const float *ga = k < 3 ? gae : gam;
      const int a = k % 3;
      size_t pts[4] = {id, id, id, id};
      int npt;
      bool ok = true;
      if (k < 3)
      {
        npt = 2;
        ok = pos[a] + 1 < lim[a];
        pts[1] = id + stride[a];
      }
      else
      {
        const int lo = a == 0 ? 1 : 0;
        const int hi = a == 2 ? 1 : 2;
        npt = 4;
        ok = pos[lo] + 1 < lim[lo] && pos[hi] + 1 < lim[hi];
        pts[1] = id + stride[hi];
        pts[2] = id + stride[lo];
        pts[3] = id + stride[lo] + stride[hi];
      }
      if (!ok)
        continue;
      bool any = false;
      for (int j = 0; j < npt; ++j)
        any = any || om[pts[j]] != 0.f || ga[pts[j]] != 0.f;
      if (any)
        f |= 1u << k;
    }
    flags[id] = (unsigned char) f;
  }
}

}  // namespace

template <int R, int W>
void launch_shape (const FusedParams &p, int *err, cudaStream_t s)
{
  const int ny = p.g.n[1], nz = p.g.n[2], nx = p.g.n[0];
  dim3 block (32, W);
  dim3 grid ((nz - 2 + 30) / 31, (ny - 2 + R * W - 2) / (R * W - 1), (nx - 2 + p.x_chunk - 1) / p.x_chunk);
  if (p.use_meta)
  {
    if (p.fp16)
      fused3d_kernel<__half, R, W, true><<<grid, block, 0, s>>> (p, err);
    else
      fused3d_kernel<float, R, W, true><<<grid, block, 0, s>>> (p, err);
  }
  else
  {
    if (p.fp16)
      fused3d_kernel<__half, R, W, false><<<grid, block, 0, s>>> (p, err);
    else
      fused3d_kernel<float, R, W, false><<<grid, block, 0, s>>> (p, err);
  }
}

// rows per CTA for each shape (R * W - 1 owned)
int fused_rows_per_cta (int shape)
{
  switch (shape)
  {
    case 0: return 4 * 4 - 1;
    case 1: return 4 * 8 - 1;
    case 2: return 8 * 4 - 1;
    case 3: return 2 * 8 - 1;
    default: return 6 * 4 - 1;
  }
}

int launch_fused3d (const FusedParams &p, int *err, cudaStream_t s)
{
  switch (p.shape)
  {
    case 0: launch_shape<4, 4> (p, err, s); break;
    case 1: launch_shape<4, 8> (p, err, s); break;
    case 2: launch_shape<8, 4> (p, err, s); break;
    case 3: launch_shape<2, 8> (p, err, s); break;
    default: launch_shape<6, 4> (p, err, s); break;
  }
  return 1;
}

namespace {

// Bounding box of the cells with any Drude flag: box[0..2] = lowest x, y, z
// (atomicMin from INT_MAX), box[3..5] = highest (atomicMax from -1).
__global__ void drude_box_kernel (const unsigned char *flags, int nx, int ny, int nz, int *box)
{
  const size_t n = (size_t) nx * ny * nz;
  int lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {-1, -1, -1};
  for (size_t id = (size_t) blockIdx.x * blockDim.x + threadIdx.x; id < n; id += (size_t) gridDim.x * blockDim.x)
  {
    if (!flags[id])
      continue;
    const int pos[3] = {(int) (id / ((size_t) ny * nz)), (int) ((id / nz) % ny), (int) (id % nz)};
    for (int a = 0; a < 3; ++a)
    {
      lo[a] = min (lo[a], pos[a]);
      hi[a] = max (hi[a], pos[a]);
    }
  }
  for (int a = 0; a < 3; ++a)
  {
    for (int o = 16; o > 0; o >>= 1)
    {
      lo[a] = min (lo[a], __shfl_xor_sync (0xffffffffu, lo[a], o));
      hi[a] = max (hi[a], __shfl_xor_sync (0xffffffffu, hi[a], o));
    }
    if ((threadIdx.x & 31) == 0 && hi[a] >= 0)
    {
      atomicMin (box + a, lo[a]);
      atomicMax (box + 3 + a, hi[a]);
    }
  }
}

// Drude fix-up after a TMA sweep step, which updates every cell with the
// plain (or PML) rule.  E pass: the Drude components of the cells of the box
// are recomputed from the old buffers with update_drude (curl of H_old, the
// sweep's operation order).  H pass, after it, over the box moved out by one
// cell on the low sides (every H cell whose curl reads an E value of the
// box): H_new recomputed from H_old and the corrected E_new with the rule of
// the cell (Drude, PML or plain).  The box holds no point source, no PML
// cell and no TF/SF band cell (the host checks), so no other rule applies.
template <typename T>
__global__ void __launch_bounds__ (256) drude_fix_e_kernel (const __grid_constant__ FusedParams p, DrudeBox b)
{
  const int ny = p.g.n[1], nz = p.g.n[2];
  const size_t sx = (size_t) ny * nz;
  const int ez = b.hi[2] - b.lo[2], ey = b.hi[1] - b.lo[1];
  const long long total = (long long) (b.hi[0] - b.lo[0]) * ey * ez;
  const T *Ho0 = (const T *) p.h_old[0], *Ho1 = (const T *) p.h_old[1], *Ho2 = (const T *) p.h_old[2];
  for (long long t = (long long) blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long) gridDim.x * blockDim.x)
  {
    const int z = b.lo[2] + (int) (t % ez);
    const int y = b.lo[1] + (int) ((t / ez) % ey);
    const int x = b.lo[0] + (int) (t / ((long long) ez * ey));
    const size_t id = (size_t) x * sx + (size_t) y * nz + z;
    const unsigned fl = p.dflag[id];
    if (!(fl & 7u))
      continue;
    if (fl & 1u)
    {
      const float c = (ldf (Ho2, id) - ldf (Ho2, id - nz)) - (ldf (Ho1, id) - ldf (Ho1, id - 1));
      stf ((T *) p.e_new[0], id, update_drude (p, 0, ldf ((const T *) p.e_old[0], id), c, x, y, z, id, true));
    }
    if (fl & 2u)
    {
      const float c = (ldf (Ho0, id) - ldf (Ho0, id - 1)) - (ldf (Ho2, id) - ldf (Ho2, id - sx));
      stf ((T *) p.e_new[1], id, update_drude (p, 1, ldf ((const T *) p.e_old[1], id), c, x, y, z, id, true));
    }
    if (fl & 4u)
    {
      const float c = (ldf (Ho1, id) - ldf (Ho1, id - sx)) - (ldf (Ho0, id) - ldf (Ho0, id - nz));
      stf ((T *) p.e_new[2], id, update_drude (p, 2, ldf ((const T *) p.e_old[2], id), c, x, y, z, id, true));
    }
  }
}

// E_new values the H pass reads were written by the E pass (or the sweep)
// before this launch, so plain loads (not the read-only path) are used.
template <typename T>
__device__ __forceinline__ float ld_new (const T *p, size_t i);
template <>
__device__ __forceinline__ float ld_new<float> (const float *p, size_t i)
{
  return p[i];
}
template <>
__device__ __forceinline__ float ld_new<__half> (const __half *p, size_t i)
{
  return __half2float (p[i]);
}

template <typename T>
__global__ void __launch_bounds__ (256) drude_fix_h_kernel (const __grid_constant__ FusedParams p, DrudeBox b)
{
  const int ny = p.g.n[1], nz = p.g.n[2];
  const size_t sx = (size_t) ny * nz;
  const int ez = b.hi[2] - b.lo[2], ey = b.hi[1] - b.lo[1];
  const long long total = (long long) (b.hi[0] - b.lo[0]) * ey * ez;
  const T *E0 = (const T *) p.e_new[0], *E1 = (const T *) p.e_new[1], *E2 = (const T *) p.e_new[2];
  for (long long t = (long long) blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long) gridDim.x * blockDim.x)
  {
    const int z = b.lo[2] + (int) (t % ez);
    const int y = b.lo[1] + (int) ((t / ez) % ey);
    const int x = b.lo[0] + (int) (t / ((long long) ez * ey));
    const size_t id = (size_t) x * sx + (size_t) y * nz + z;
    const unsigned fl = p.dflag[id];
    const float ex = ld_new (E0, id), ey_ = ld_new (E1, id), ez_ = ld_new (E2, id);
    const float a = (ld_new (E1, id + 1) - ey_) - (ld_new (E2, id + nz) - ez_);
    const float bb = (ld_new (E2, id + sx) - ez_) - (ld_new (E0, id + 1) - ex);
    const float c = (ld_new (E0, id + nz) - ex) - (ld_new (E1, id + sx) - ey_);
    auto inside = [&] (int k) {
      return x >= p.ilo[k][0] && x < p.ihi[k][0] && y >= p.ilo[k][1] && y < p.ihi[k][1] && z >= p.ilo[k][2] &&
             z < p.ihi[k][2];
    };
    const float h0 = update_any<3, true> (p, fl, inside (3), ldf ((const T *) p.h_old[0], id), a, 1.f, x, y, z, id,
                                          true);
    const float h1 = update_any<4, true> (p, fl, inside (4), ldf ((const T *) p.h_old[1], id), bb, 1.f, x, y, z, id,
                                          true);
    const float h2 = update_any<5, true> (p, fl, inside (5), ldf ((const T *) p.h_old[2], id), c, 1.f, x, y, z, id,
                                          true);
    stf ((T *) p.h_new[0], id, h0);
    stf ((T *) p.h_new[1], id, h1);
    stf ((T *) p.h_new[2], id, h2);
  }
}

}  // namespace

int launch_drude_box (const unsigned char *flags, int nx, int ny, int nz, int *box, cudaStream_t s)
{
  const int init[6] = {INT_MAX, INT_MAX, INT_MAX, -1, -1, -1};
  if (cudaMemcpyAsync (box, init, sizeof (init), cudaMemcpyHostToDevice, s) != cudaSuccess)
    return 0;
  size_t n = (size_t) nx * ny * nz;
  size_t blocks = (n + 255) / 256;
  if (blocks > 148 * 16)
    blocks = 148 * 16;
  drude_box_kernel<<<(unsigned) blocks, 256, 0, s>>> (flags, nx, ny, nz, box);
  return 1;
}

int launch_drude_fixup (const FusedParams &p, const DrudeBox &box, cudaStream_t s)
{
  DrudeBox hb = box;   // H pass: one more cell on the low sides, within the updated cells
  for (int a = 0; a < 3; ++a)
    hb.lo[a] = max (box.lo[a] - 1, 1);
  auto blocks = [] (const DrudeBox &b) {
    long long n = 1;
    for (int a = 0; a < 3; ++a)
      n *= b.hi[a] - b.lo[a];
    return (unsigned) std::min<long long> ((n + 255) / 256, 148 * 16);
  };
  if (p.fp16)
  {
    drude_fix_e_kernel<__half><<<blocks (box), 256, 0, s>>> (p, box);
    drude_fix_h_kernel<__half><<<blocks (hb), 256, 0, s>>> (p, hb);
  }
  else
  {
    drude_fix_e_kernel<float><<<blocks (box), 256, 0, s>>> (p, box);
    drude_fix_h_kernel<float><<<blocks (hb), 256, 0, s>>> (p, hb);
  }
  return 2;
}

__global__ void current_fix_kernel (FusedParams p, CurrentFix cf, const double *src)
{
  if (threadIdx.x != 0 || blockIdx.x != 0)
    return;
  const int ny = p.g.n[1], nz = p.g.n[2];
  const size_t st[3] = {(size_t) ny * nz, (size_t) nz, 1};
  const size_t c = (size_t) cf.pos[0] * st[0] + (size_t) cf.pos[1] * st[1] + cf.pos[2];
  const float S = p.courant;
  auto rmw = [&] (void *f, size_t id, float d) {
    if (p.fp16)
    {
      __half *h = static_cast<__half *> (f);
      h[id] = __float2half_rn (__half2float (h[id]) + d);
    }
    else
      static_cast<float *> (f)[id] += d;
  };
  // H at cell q: the update adds S times its curl; a change dE of E
  // component k at c changes the curls of the two other H components
  // (E_CENTERED: Hx = (Ey(z+1) - Ey) - (Ez(y+1) - Ez), and its rotations)
  auto h_at = [&] (int m, int dax, float d) {
    // H component m at c - e_dax (dax = -1: at c itself) takes S d
    int q[3] = {cf.pos[0], cf.pos[1], cf.pos[2]};
    if (dax >= 0)
      q[dax] -= 1;
    for (int a = 0; a < 3; ++a)
      if (!((p.g.drop >> a) & 1) && (q[a] < 1 || q[a] > p.g.n[a] - 2))
        return;   // a face cell: the step does not update it
    rmw (p.h_new[m], (size_t) q[0] * st[0] + (size_t) q[1] * st[1] + q[2], S * d);
  };
  const float ie = (float) (src[0] * p.g.dx) * cf.scale_e;
  for (int k = 0; k < 3; ++k)
  {
    if (!((cf.mask_e >> k) & 1))
      continue;
    const float im = p.eps ? __fdividef (2.f, p.eps[c] + p.eps[c + st[k]]) : 1.f;
    const float de = S * im * -ie;
    rmw (p.e_new[k], c, de);
    // the two H components whose curl holds E_k: m = k + 1 and k + 2 (mod 3)
    const int m1 = (k + 1) % 3, m2 = (k + 2) % 3;
    // H_m1 reads E_k along axis m2 with sign -, H_m2 reads it along m1 with sign +
    // (Hx: +dz Ey - dy Ez; Hy: +dx Ez - dz Ex; Hz: +dy Ex - dx Ey)
    h_at (m1, -1, de);
    h_at (m1, m2, -de);
    h_at (m2, -1, -de);
    h_at (m2, m1, de);
  }
  const float ih = (float) (src[1] * p.g.dx) * cf.scale_h;
  for (int m = 0; m < 3; ++m)
    if ((cf.mask_h >> m) & 1)
      rmw (p.h_new[m], c, S * -ih);
}

int launch_current_fix (const FusedParams &p, const CurrentFix &cf, const double *src, cudaStream_t s)
{
  current_fix_kernel<<<1, 32, 0, s>>> (p, cf, src);
  return 1;
}

int launch_drude_flags (unsigned char *flags, const float *ome, const float *gae, const float *omm, const float *gam,
                        int nx, int ny, int nz, cudaStream_t s)
{
  size_t n = (size_t) nx * ny * nz;
  size_t blocks = (n + 255) / 256;
  if (blocks > 148 * 32)
    blocks = 148 * 32;
  drude_flags_kernel<<<(unsigned) blocks, 256, 0, s>>> (flags, ome, gae, omm, gam, nx, ny, nz);
  return 1;
}

}  // namespace fdtdb
