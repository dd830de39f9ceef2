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

template <typename T, int TY, int TZ, bool META, int MINB>
__global__ void __launch_bounds__ ((TY + 1) * (TZ + 1), MINB) fused3d_kernel (FusedParams p, int *err)
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
  const bool halo_y = ty == 0 && z <= nz - 1;              // loads (y - 1) for Hx, Hz
  const bool halo_z = tz == 0 && y <= ny - 1;              // loads (z - 1) for Hx, Hy
  const bool ring_y = ty == TY && p.eps && y + 1 <= ny - 1 && z <= nz - 1;
  const bool ring_z = tz == TZ && p.eps && z + 1 <= nz - 1 && y <= ny - 1;

  __shared__ float sH[3][TY + 2][TZ + 2];
  __shared__ float sE[3][TY + 1][TZ + 1];
  __shared__ float sEps[TY + 2][TZ + 2];

  bool yz_in[6];
#pragma unroll
  for (int k = 0; k < 6; ++k)
    yz_in[k] = !p.use_pml || (y >= p.ilo[k][1] && y < p.ihi[k][1] && z >= p.ilo[k][2] && z < p.ihi[k][2]);
  const bool yz_face = p.use_tfsf && (on_face (p.face[1], y) || on_face (p.face[2], z));

  const T *Eo0 = (const T *) p.e_old[0], *Eo1 = (const T *) p.e_old[1], *Eo2 = (const T *) p.e_old[2];
  const T *Ho0 = (const T *) p.h_old[0], *Ho1 = (const T *) p.h_old[1], *Ho2 = (const T *) p.h_old[2];
  T *En0 = (T *) p.e_new[0], *En1 = (T *) p.e_new[1], *En2 = (T *) p.e_new[2];
  T *Hn0 = (T *) p.h_new[0], *Hn1 = (T *) p.h_new[1], *Hn2 = (T *) p.h_new[2];

  // registers of the plane being fetched (software pipeline, one plane ahead)
  float fh0 = 0.f, fh1 = 0.f, fh2 = 0.f, fe0 = 0.f, fe1 = 0.f, fe2 = 0.f;
  float feps = 1.f, feps1 = 1.f, fhy0 = 0.f, fhy2 = 0.f, fhz0 = 0.f, fhz1 = 0.f, fry = 1.f, frz = 1.f;
  unsigned ffl = 0;
  auto fetch = [&] (int x) {
    const size_t id = (size_t) x * sx + col;
    if (valid)
    {
      fh0 = ldf (Ho0, id);
      fh1 = ldf (Ho1, id);
      fh2 = ldf (Ho2, id);
      fe0 = ldf (Eo0, id);
      fe1 = ldf (Eo1, id);
      fe2 = ldf (Eo2, id);
      if (p.eps)
      {
        feps = __ldg (p.eps + id);
        feps1 = x + 1 <= nx - 1 ? __ldg (p.eps + id + sx) : 1.f;
      }
      if (META)
        ffl = p.dflag[id];
    }
    if (halo_y)
    {
      fhy0 = ldf (Ho0, id - nz);
      fhy2 = ldf (Ho2, id - nz);
    }
    if (halo_z)
    {
      fhz0 = ldf (Ho0, id - 1);
      fhz1 = ldf (Ho1, id - 1);
    }
    if (ring_y)
      fry = __ldg (p.eps + id + nz);
    if (ring_z)
      frz = __ldg (p.eps + id + 1);
  };

  float hp0 = 0.f, hp1 = 0.f, hp2 = 0.f;   // H_old(x - 1), own cell
  float ep0 = 0.f, ep1 = 0.f, ep2 = 0.f;   // E_new(x - 1), own cell
  unsigned flp = 0;
  if (valid)
  {
    const size_t id = (size_t) (xa - 1) * sx + col;
    hp0 = ldf (Ho0, id);
    hp1 = ldf (Ho1, id);
    hp2 = ldf (Ho2, id);
    if (META)
      flp = p.dflag[id];
  }
  fetch (xa);

  for (int x = xa; x <= xb + 1; ++x)
  {
    const size_t id = (size_t) x * sx + col;
    // 1. stage the fetched plane
    sH[0][ty + 1][tz + 1] = fh0;
    sH[1][ty + 1][tz + 1] = fh1;
    sH[2][ty + 1][tz + 1] = fh2;
    sEps[ty][tz] = feps;
    if (ty == 0)
    {
      sH[0][0][tz + 1] = fhy0;
      sH[2][0][tz + 1] = fhy2;
    }
    if (tz == 0)
    {
      sH[0][ty + 1][0] = fhz0;
      sH[1][ty + 1][0] = fhz1;
    }
    if (ty == TY)
      sEps[TY + 1][tz] = fry;
    if (tz == TZ)
      sEps[ty][TZ + 1] = frz;
    const float eo0 = fe0, eo1 = fe1, eo2 = fe2;
    const float epsx1 = feps1;
    const unsigned fl = ffl;
    const float h0 = fh0, h1 = fh1, h2 = fh2;
    __syncthreads ();
    // 2. next plane in flight while this one computes
    if (x + 1 <= xb + 1)
      fetch (x + 1);

    // 3. E_new(x) on tile + ring
    float en0 = eo0, en1 = eo1, en2 = eo2;
    if (inner && x <= nx - 2)
    {
      float i0 = 1.f, i1 = 1.f, i2 = 1.f;
      if (p.eps)
      {
        const float e0 = sEps[ty][tz];
        i0 = __fdividef (2.f, e0 + epsx1);
        i1 = __fdividef (2.f, e0 + sEps[ty + 1][tz]);
        i2 = __fdividef (2.f, e0 + sEps[ty][tz + 1]);
      }
      // Ex: Hz(y-1), Hz, Hy(z-1), Hy ; Ey: Hx(z-1), Hx, Hz(x-1), Hz ; Ez: Hy(x-1), Hy, Hx(y-1), Hx
      float a0 = sH[2][ty][tz + 1], a1 = h2, a2 = sH[1][ty + 1][tz], a3 = h1;
      float b0 = sH[0][ty + 1][tz], b1 = h0, b2 = hp2, b3 = h2;
      float c0 = hp1, c1 = h1, c2 = sH[0][ty][tz + 1], c3 = h0;
      if (yz_face || (p.use_tfsf && on_face (p.face[0], x)))
      {
        tfsf_apply (p, 0, p.inc_h, err, x, y, z, a0, a1, a2, a3);
        tfsf_apply (p, 1, p.inc_h, err, x, y, z, b0, b1, b2, b3);
        tfsf_apply (p, 2, p.inc_h, err, x, y, z, c0, c1, c2, c3);
      }
      const bool st = owner && x <= xb;
      en0 = update_any<0, META> (p, fl, yz_in[0] && x >= p.ilo[0][0] && x < p.ihi[0][0], eo0, (a1 - a0) - (a3 - a2),
                                 i0, x, y, z, id, st);
      en1 = update_any<1, META> (p, fl, yz_in[1] && x >= p.ilo[1][0] && x < p.ihi[1][0], eo1, (b1 - b0) - (b3 - b2),
                                 i1, x, y, z, id, st);
      en2 = update_any<2, META> (p, fl, yz_in[2] && x >= p.ilo[2][0] && x < p.ihi[2][0], eo2, (c1 - c0) - (c3 - c2),
                                 i2, x, y, z, id, st);
      if ((p.ps_mask & 7) && x == p.ps[0] && y == p.ps[1] && z == p.ps[2])
      {
        const float v = (float) p.src[p.src_index];
        if (p.ps_mask & 1)
          en0 = v;
        if (p.ps_mask & 2)
          en1 = v;
        if (p.ps_mask & 4)
          en2 = v;
      }
      if (st)
      {
        stf (En0, id, en0);
        stf (En1, id, en1);
        stf (En2, id, en2);
      }
    }

    // 4. H_new(x - 1) on the tile
    const int xh = x - 1;
    if (owner && xh >= xa)
    {
      const size_t hid = id - sx;
      // Hx: Ey, Ey(z+1), Ez, Ez(y+1) ; Hy: Ez, Ez(x+1), Ex, Ex(z+1) ; Hz: Ex, Ex(y+1), Ey, Ey(x+1)
      float a0 = ep1, a1 = sE[1][ty][tz + 1], a2 = ep2, a3 = sE[2][ty + 1][tz];
      float b0 = ep2, b1 = en2, b2 = ep0, b3 = sE[0][ty][tz + 1];
      float c0 = ep0, c1 = sE[0][ty + 1][tz], c2 = ep1, c3 = en1;
      if (yz_face || (p.use_tfsf && on_face (p.face[0], xh)))
      {
        tfsf_apply (p, 3, p.inc_e, err, xh, y, z, a0, a1, a2, a3);
        tfsf_apply (p, 4, p.inc_e, err, xh, y, z, b0, b1, b2, b3);
        tfsf_apply (p, 5, p.inc_e, err, xh, y, z, c0, c1, c2, c3);
      }
      float hn0 = update_any<3, META> (p, flp, yz_in[3] && xh >= p.ilo[3][0] && xh < p.ihi[3][0], hp0,
                                       (a1 - a0) - (a3 - a2), 1.f, xh, y, z, hid, true);
      float hn1 = update_any<4, META> (p, flp, yz_in[4] && xh >= p.ilo[4][0] && xh < p.ihi[4][0], hp1,
                                       (b1 - b0) - (b3 - b2), 1.f, xh, y, z, hid, true);
      float hn2 = update_any<5, META> (p, flp, yz_in[5] && xh >= p.ilo[5][0] && xh < p.ihi[5][0], hp2,
                                       (c1 - c0) - (c3 - c2), 1.f, xh, y, z, hid, true);
      if ((p.ps_mask & 56) && xh == p.ps[0] && y == p.ps[1] && z == p.ps[2])
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
    __syncthreads ();

    // 5. carry plane x into the next iteration
    sE[0][ty][tz] = valid ? en0 : 0.f;
    sE[1][ty][tz] = valid ? en1 : 0.f;
    sE[2][ty][tz] = valid ? en2 : 0.f;
    ep0 = en0;
    ep1 = en1;
    ep2 = en2;
    hp0 = h0;
    hp1 = h1;
    hp2 = h2;
    flp = fl;
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

template <int TY, int MINB>
void launch_shape (const FusedParams &p, int *err, cudaStream_t s)
{
  constexpr int TZ = 32;
  const int ny = p.g.n[1], nz = p.g.n[2], nx = p.g.n[0];
  dim3 block (TZ + 1, TY + 1);
  dim3 grid ((nz - 2 + TZ - 1) / TZ, (ny - 2 + TY - 1) / TY, (nx - 2 + p.x_chunk - 1) / p.x_chunk);
  if (p.use_meta)
  {
    if (p.fp16)
      fused3d_kernel<__half, TY, TZ, true, MINB><<<grid, block, 0, s>>> (p, err);
    else
      fused3d_kernel<float, TY, TZ, true, MINB><<<grid, block, 0, s>>> (p, err);
  }
  else
  {
    if (p.fp16)
      fused3d_kernel<__half, TY, TZ, false, MINB><<<grid, block, 0, s>>> (p, err);
    else
      fused3d_kernel<float, TY, TZ, false, MINB><<<grid, block, 0, s>>> (p, err);
  }
}

int launch_fused3d (const FusedParams &p, int *err, cudaStream_t s)
{
  switch (p.shape)
  {
    case 0: launch_shape<8, 2> (p, err, s); break;
    case 1: launch_shape<8, 3> (p, err, s); break;
    case 2: launch_shape<4, 4> (p, err, s); break;
    case 3: launch_shape<16, 1> (p, err, s); break;
    default: launch_shape<4, 6> (p, err, s); break;
  }
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
