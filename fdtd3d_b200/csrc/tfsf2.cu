// tfsf2.cu - TF/SF corrections of a pair of time steps taken by the
// two-step sweep.
//
// The two-step sweep advances a pair of steps without the TF/SF corrections.
// The corrections are linear in the fields and enter each step as changes of
// the curls on the cells of the TF/SF terms (InternalScheme.inc.h:1386-1835):
// dE(t) on E cells (from the incident H before the step's H update) and
// dH(t) on H cells (from the incident E after the step's E update).  So the
// corrected pair is the uncorrected pair plus the response to them:
//   dE1 = S im dE(t1)                     dH1 = S (curlH dE1 + dH(t1))
//   dE2 = dE1 + S im (curlE dH1 + dE(t2)) dH2 = dH1 + S (curlH dE2 + dH(t2))
// with curlH / curlE the step's own curls (E at c and c + e_a for H, H at c
// and c - e_a for E).  One kernel evaluates the four in shared memory, tile
// by tile: a tile owns a box of the support of dH2 (the TF/SF term boxes
// grown by up to two cells, which holds the support of dE2) and recomputes
// the intermediate corrections over a halo of one cell below and two above;
// only the fields of its own cells are read and written in HBM (E += dE2,
// H += dH2).  Every cell of the supports takes the plain update in both
// steps (no PML, no point source), which the host checks.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "incident_dev.cuh"
#include "tfsf2.h"

namespace fdtdb {

namespace {

template <typename T>
__device__ __forceinline__ float ldf (const T *p, size_t i);
template <>
__device__ __forceinline__ float ldf<float> (const float *p, size_t i)
{
  return p[i];
}
template <>
__device__ __forceinline__ float ldf<__half> (const __half *p, size_t i)
{
  return __half2float (p[i]);
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

// TF/SF change of the curl of a component at a cell from one of its terms:
// the incident value at distance d along the wave (linear interpolation of
// the 1-D incident grid, as inc_at), times pp (the incident component's
// projection and the term's sign, in FP64), rounded to float and times ss
// (the component's incident scale and the sign of the curl neighbour the
// term modifies, (n1 - n0) - (n3 - n2)), as the single-step kernels'
// tfsf_curl does.
__device__ __forceinline__ float term_at (const double *inc, int inc_len, int *err, double d, double pp, float ss)
{
  const int i1 = (int) d;
  const double pr2 = d - (double) i1;
  if (i1 < 0 || i1 + 1 >= inc_len)
  {
    *err = 1;
    return 0.f;
  }
  return (float) ((inc[i1] * (1 - pr2) + inc[i1 + 1] * pr2) * pp) * ss;
}

// q / d for 0 <= q < 2^22 and 1 <= d < 2^11 (rd = 1 / d rounded): the
// float quotient is off by at most one, which the remainder corrects.
__device__ __forceinline__ int small_div (int q, int d, float rd)
{
  int x = __float2int_rz (__int2float_rn (q) * rd);
  const int r = q - x * d;
  return x + (r >= d) - (r < 0);
}

// The cells of an X x Y x Z box, z fastest, strided over the CTA's threads
// (q = (x Y + y) Z + z); one decomposition at the start, carries after it.
struct Walk
{
  int q, x, y, z, Y, Z, dx, dy, dz;
  __device__ Walk (int Yd, int Zd) : Y (Yd), Z (Zd)
  {
    const float rY = __frcp_rn ((float) Y), rZ = __frcp_rn ((float) Z);
    q = threadIdx.x;
    int a = small_div (q, Z, rZ);
    z = q - a * Z;
    x = small_div (a, Y, rY);
    y = a - x * Y;
    const int s = blockDim.x;
    a = small_div (s, Z, rZ);
    dz = s - a * Z;
    dx = small_div (a, Y, rY);
    dy = a - dx * Y;
  }
  __device__ void next ()
  {
    q += blockDim.x;
    z += dz;
    int c = z >= Z;
    z -= c ? Z : 0;
    y += dy + c;
    c = y >= Y;
    y -= c ? Y : 0;
    x += dx + c;
  }
};

// One tile: own box O = [lo, hi).  Shared memory holds, per axis, the E
// corrections over D_E = [lo - 1, hi + 2), the H corrections over
// D_H = [lo - 1, hi + 1) (three components each) and eps over
// [lo - 1, hi + 3) (im = 2 / (eps + eps') of an E component at c reads eps
// at c and c + e_k).  Both correction arrays start at zero.  Each step's
// correction is its curl part, computed over the tile's phase box (where it
// can be nonzero: the supports are slabs a few cells thick), plus its TF/SF
// terms, added term by term over the cells of each term's box only:
//   1. dE1 = S im dE(t1)                                  (terms only)
//   2. dH1 = S curlH dE1 + S dH(t1)            (E at c, c + e_a: in D_E)
//   3. dE2 = dE1 + S im curlE dH1 + S im dE(t2), in place (H at c, c - e_a)
//   4. dH2 = dH1 + S curlH dE2 + S dH(t2) over O; the fields of O take
//      E += dE2 and H += dH2 where nonzero.
template <typename T>
__global__ void __launch_bounds__ (256, 4) tfsf2_fused (const __grid_constant__ FusedParams p, const Tf2Tile *tiles,
                                                        const double *inc_h1, const double *inc_e1,
                                                        const double *inc_h2, const double *inc_e2, int *err)
{
  extern __shared__ float tf_smem[];
  const Tf2Tile &t = tiles[blockIdx.x];
  const unsigned mask = t.mask;
  const int ex = t.hi[0] - t.lo[0], ey = t.hi[1] - t.lo[1], ez = t.hi[2] - t.lo[2];
  const int eY = ey + 3, eZ = ez + 3, nE = (ex + 3) * eY * eZ, dEx = eY * eZ;
  const int hY = ey + 2, hZ = ez + 2, nH = (ex + 2) * hY * hZ, dHx = hY * hZ;
  const int pY = ey + 4, pZ = ez + 4, nP = (ex + 4) * pY * pZ;
  float *const sE = tf_smem;
  float *const sH = sE + 3 * nE;
  float *const sP = sH + 3 * nH;
  const int nx = p.g.n[0], ny = p.g.n[1], nz = p.g.n[2];
  const size_t sx = (size_t) ny * nz, sy = nz;
  const float S = p.courant;
  const int o[3] = {t.lo[0] - 1, t.lo[1] - 1, t.lo[2] - 1};   // origin of every domain
  const bool has_eps = p.eps != nullptr;
  // term (k, t) of the tile, entry 4 k + t: the incident distance at local
  // cell q is d = A qx + B qy + C qz + tD (tD folds the tile origin, the
  // term's neighbour offset, the incident component's position and the half
  // cell of the H components), its value term_at (.., d, tP, tS)
  __shared__ double tD[24], tP[24];
  __shared__ float tS[24];
  const double A = p.g.s1 * p.g.c2, B = p.g.s1 * p.g.s2, C = p.g.c1;
  if (threadIdx.x < 24)
  {
    const int k = threadIdx.x >> 2, tt = threadIdx.x & 3;
    if (tt < p.comp[k].nterms)
    {
      const TermDev &tm = p.comp[k].term[tt];
      const int ic = tm.inc_comp;
      const double x0 = ((double) (o[0] + tm.aux[0]) + p.g.min_fp[ic][0]) - p.g.zero_inc[0];
      const double y0 = ((double) (o[1] + tm.aux[1]) + p.g.min_fp[ic][1]) - p.g.zero_inc[1];
      const double z0 = ((double) (o[2] + tm.aux[2]) + p.g.min_fp[ic][2]) - p.g.zero_inc[2];
      tD[threadIdx.x] = A * x0 + B * y0 + C * z0 - (ic >= 3 ? 0.5 : 0.0);
      tP[threadIdx.x] = p.g.proj[ic] * tm.negate;
      tS[threadIdx.x] = (tm.slot == 0 || tm.slot == 3) ? p.inc_scale[ic] : -p.inc_scale[ic];
    }
  }

  // zero corrections (both arrays: 3 (nE + nH) floats, sE 16-byte aligned)
  {
    const int n4 = 3 * (nE + nH) / 4;
    float4 *z4 = reinterpret_cast<float4 *> (sE);
    for (int i = threadIdx.x; i < n4; i += blockDim.x)
      z4[i] = make_float4 (0.f, 0.f, 0.f, 0.f);
    for (int i = 4 * n4 + threadIdx.x; i < 3 * (nE + nH); i += blockDim.x)
      sE[i] = 0.f;
  }
  // eps where S im is taken: the E term cells (phase box 0) and the dE2
  // curl cells (phase box 2), each with its +1 neighbours (indices clamped
  // to the grid: only cells of the supports, two cells inside the faces,
  // use it)
  if (has_eps)
  {
    int b0[3], b1[3];
    bool any = true;
#pragma unroll
    for (int a = 0; a < 3; ++a)
    {
      const bool e0 = t.ph[0][a] >= t.ph[0][3 + a], e2 = t.ph[2][a] >= t.ph[2][3 + a];
      any = any && !(e0 && e2);
      b0[a] = e0 ? t.ph[2][a] : (e2 ? t.ph[0][a] : min (t.ph[0][a], t.ph[2][a]));
      b1[a] = (e0 ? t.ph[2][3 + a] : (e2 ? t.ph[0][3 + a] : max (t.ph[0][3 + a], t.ph[2][3 + a]))) + 1;
    }
    if (any)
    {
      const int bY = b1[1] - b0[1], bZ = b1[2] - b0[2], nb = (b1[0] - b0[0]) * bY * bZ;
      for (Walk w (bY, bZ); w.q < nb; w.next ())
      {
        const int qx = b0[0] + w.x, qy = b0[1] + w.y, qz = b0[2] + w.z;
        const int x = min (o[0] + qx, nx - 1), y = min (o[1] + qy, ny - 1), z = min (o[2] + qz, nz - 1);
        sP[(qx * pY + qy) * pZ + qz] = p.eps[(size_t) x * sx + (size_t) y * sy + z];
      }
    }
  }
  __syncthreads ();
  // S im of E component k at domain cell (qx, qy, qz)
  auto s_im = [&] (int k, int qx, int qy, int qz) -> float {
    if (!has_eps)
      return S;
    const int q = (qx * pY + qy) * pZ + qz;
    const int st = k == 0 ? pY * pZ : (k == 1 ? pZ : 1);
    return S * __fdividef (2.f, sP[q] + sP[q + st]);
  };
  // the TF/SF terms of the family kb .. kb + 2 (E: 0, H: 3) over the cells
  // of the local domain d0 .. d1 - 1: for each cell of a term's box,
  // add (k - kb, cell, term value).  Pass j takes every component's j-th
  // term (the components write their own arrays, so a pass adds to a cell
  // of an array at most once); the CTA synchronises after each pass (two
  // terms of a component may share a cell).  The cells of a pass's boxes
  // form one index range strided over the threads, two cells an iteration,
  // so that the incident-grid loads of both are in flight at once.
  auto terms = [&] (int kb, const double *inc, int d0, const int d1[3], auto &&add) {
    unsigned mk[3];
    int passes = 0;
#pragma unroll
    for (int c = 0; c < 3; ++c)
    {
      mk[c] = (mask >> (4 * (kb + c))) & 15u;
      passes = max (passes, __popc (mk[c]));
    }
#pragma unroll 1
    for (int j = 0; j < passes; ++j)
    {
      // component c's box: cells bl[c] + (0 .. bX, 0 .. bY[c], 0 .. bZ[c]), n[c] of them
      int n[3], tt[3], bl[3][3], bY[3], bZ[3];
      float rY[3], rZ[3];
#pragma unroll
      for (int c = 0; c < 3; ++c)
      {
        n[c] = 0;
        tt[c] = 0;
        bY[c] = 1;
        bZ[c] = 1;
        rY[c] = 1.f;
        rZ[c] = 1.f;
        bl[c][0] = bl[c][1] = bl[c][2] = 0;
        if (!mk[c])
          continue;
        tt[c] = __ffs (mk[c]) - 1;
        mk[c] &= mk[c] - 1;
        const TermDev &tm = p.comp[kb + c].term[tt[c]];
        int ext[3];
#pragma unroll
        for (int a = 0; a < 3; ++a)
        {
          bl[c][a] = max (tm.lo[a] - o[a], d0);
          ext[a] = min (tm.hi[a] - o[a], d1[a]) - bl[c][a];
        }
        if (ext[0] > 0 && ext[1] > 0 && ext[2] > 0)
        {
          n[c] = ext[0] * ext[1] * ext[2];
          bY[c] = ext[1];
          bZ[c] = ext[2];
          rY[c] = __frcp_rn ((float) ext[1]);
          rZ[c] = __frcp_rn ((float) ext[2]);
        }
      }
      const int n01 = n[0] + n[1], N = n01 + n[2];
      if (N == 0)
        continue;   // nothing written: no barrier needed
      // flat index f of the pass -> component c and local cell
      auto cell = [&] (int f, int &c, int &qx, int &qy, int &qz) {
        const bool a0 = f < n[0], a1 = f < n01;
        c = a0 ? 0 : (a1 ? 1 : 2);
        const int l = f - (a0 ? 0 : (a1 ? n[0] : n01));
        const int Y = a0 ? bY[0] : (a1 ? bY[1] : bY[2]), Z = a0 ? bZ[0] : (a1 ? bZ[1] : bZ[2]);
        const int q = small_div (l, Z, a0 ? rZ[0] : (a1 ? rZ[1] : rZ[2]));
        const int x = small_div (q, Y, a0 ? rY[0] : (a1 ? rY[1] : rY[2]));
        qx = x + (a0 ? bl[0][0] : (a1 ? bl[1][0] : bl[2][0]));
        qy = q - x * Y + (a0 ? bl[0][1] : (a1 ? bl[1][1] : bl[2][1]));
        qz = l - q * Z + (a0 ? bl[0][2] : (a1 ? bl[1][2] : bl[2][2]));
      };
      const int s = blockDim.x;
      for (int f = threadIdx.x; f < N; f += 2 * s)
      {
        // the second cell (f + s) is evaluated even past the range (as the
        // first again) so that both evaluations are straight-line code
        const bool two = f + s < N;
        int c0, x0, y0, z0, c1, x1, y1, z1;
        cell (f, c0, x0, y0, z0);
        cell (two ? f + s : f, c1, x1, y1, z1);
        const int e0 = 4 * (kb + c0) + (c0 == 0 ? tt[0] : (c0 == 1 ? tt[1] : tt[2]));
        const int e1 = 4 * (kb + c1) + (c1 == 0 ? tt[0] : (c1 == 1 ? tt[1] : tt[2]));
        const double d0 = fma (A, (double) x0, fma (B, (double) y0, fma (C, (double) z0, tD[e0])));
        const double d1 = fma (A, (double) x1, fma (B, (double) y1, fma (C, (double) z1, tD[e1])));
        const float v0 = term_at (inc, p.inc_len, err, d0, tP[e0], tS[e0]);
        const float v1 = term_at (inc, p.inc_len, err, d1, tP[e1], tS[e1]);
        add (c0, x0, y0, z0, v0);
        if (two)
          add (c1, x1, y1, z1, v1);
      }
      __syncthreads ();
    }
  };
  // the cells of phase box f (local x, y, z)
  auto box_walk = [&] (int f, auto &&body) {
    const int b0 = t.ph[f][0], b1 = t.ph[f][1], b2 = t.ph[f][2];
    const int bY = t.ph[f][4] - b1, bZ = t.ph[f][5] - b2, bX = t.ph[f][3] - b0;
    if (bX <= 0 || bY <= 0 || bZ <= 0)
      return;
    for (Walk w (bY, bZ); w.q < bX * bY * bZ; w.next ())
      body (b0 + w.x, b1 + w.y, b2 + w.z);
  };
  const int dE1[3] = {ex + 3, ey + 3, ez + 3}, dH1[3] = {ex + 2, ey + 2, ez + 2};
  const int dO1[3] = {ex + 1, ey + 1, ez + 1};

  // 1. dE1 on the E term cells
  terms (0, inc_h1, 0, dE1, [&] (int k, int qx, int qy, int qz, float dv) {
    sE[k * nE + (qx * eY + qy) * eZ + qz] += s_im (k, qx, qy, qz) * dv;
  });
  // 2. dH1: the curl of dE1 over its phase box, then the H terms
  {
    const float *E0 = sE, *E1 = sE + nE, *E2 = sE + 2 * nE;
    box_walk (1, [&] (int qx, int qy, int qz) {
      const int e = (qx * eY + qy) * eZ + qz, h = (qx * hY + qy) * hZ + qz;
      sH[h] = S * ((E1[e + 1] - E1[e]) - (E2[e + eZ] - E2[e]));
      sH[nH + h] = S * ((E2[e + dEx] - E2[e]) - (E0[e + 1] - E0[e]));
      sH[2 * nH + h] = S * ((E0[e + eZ] - E0[e]) - (E1[e + dEx] - E1[e]));
    });
  }
  __syncthreads ();
  terms (3, inc_e1, 0, dH1, [&] (int m, int qx, int qy, int qz, float dv) {
    sH[m * nH + (qx * hY + qy) * hZ + qz] += S * dv;
  });
  // 3. dE2: the curl of dH1 over its phase box, then the E terms (over U)
  {
    const float *H0 = sH, *H1 = sH + nH, *H2 = sH + 2 * nH;
    box_walk (2, [&] (int qx, int qy, int qz) {
      const int h = (qx * hY + qy) * hZ + qz, e = (qx * eY + qy) * eZ + qz;
      const float cu[3] = {(H2[h] - H2[h - hZ]) - (H1[h] - H1[h - 1]), (H0[h] - H0[h - 1]) - (H2[h] - H2[h - dHx]),
                           (H1[h] - H1[h - dHx]) - (H0[h] - H0[h - hZ])};
#pragma unroll
      for (int k = 0; k < 3; ++k)
        if (cu[k] != 0.f)
          sE[k * nE + e] += s_im (k, qx, qy, qz) * cu[k];
    });
  }
  __syncthreads ();
  terms (0, inc_h2, 1, dH1, [&] (int k, int qx, int qy, int qz, float dv) {
    sE[k * nE + (qx * eY + qy) * eZ + qz] += s_im (k, qx, qy, qz) * dv;
  });
  // 4. dH2 over O: the curl of dE2, then the H terms; then the fields
  {
    const float *E0 = sE, *E1 = sE + nE, *E2 = sE + 2 * nE;
    for (Walk w (ey, ez); w.q < ex * ey * ez; w.next ())
    {
      const int qx = w.x + 1, qy = w.y + 1, qz = w.z + 1;
      const int e = (qx * eY + qy) * eZ + qz, h = (qx * hY + qy) * hZ + qz;
      sH[h] += S * ((E1[e + 1] - E1[e]) - (E2[e + eZ] - E2[e]));
      sH[nH + h] += S * ((E2[e + dEx] - E2[e]) - (E0[e + 1] - E0[e]));
      sH[2 * nH + h] += S * ((E0[e + eZ] - E0[e]) - (E1[e + dEx] - E1[e]));
    }
  }
  __syncthreads ();
  terms (3, inc_e2, 1, dO1, [&] (int m, int qx, int qy, int qz, float dv) {
    sH[m * nH + (qx * hY + qy) * hZ + qz] += S * dv;
  });
  // the fields of O: all loads of a cell first, then the stores
  for (Walk w (ey, ez); w.q < ex * ey * ez; w.next ())
  {
    const int qx = w.x + 1, qy = w.y + 1, qz = w.z + 1;
    const int e = (qx * eY + qy) * eZ + qz, h = (qx * hY + qy) * hZ + qz;
    const size_t id = (size_t) (o[0] + qx) * sx + (size_t) (o[1] + qy) * sy + (o[2] + qz);
    float de[3], dh[3], fe[3], fh[3];
#pragma unroll
    for (int k = 0; k < 3; ++k)
    {
      de[k] = sE[k * nE + e];
      dh[k] = sH[k * nH + h];
      fe[k] = de[k] != 0.f ? ldf (reinterpret_cast<const T *> (p.e_new[k]), id) : 0.f;
      fh[k] = dh[k] != 0.f ? ldf (reinterpret_cast<const T *> (p.h_new[k]), id) : 0.f;
    }
#pragma unroll
    for (int k = 0; k < 3; ++k)
    {
      if (de[k] != 0.f)
        stf (reinterpret_cast<T *> (p.e_new[k]), id, fe[k] + de[k]);
      if (dh[k] != 0.f)
        stf (reinterpret_cast<T *> (p.h_new[k]), id, fh[k] + dh[k]);
    }
  }
}

// Disjoint cover of a union of boxes: coordinate compression (every box edge
// is a cut), the covered elementary boxes, runs along z merged; each box
// carries the mask of the TF/SF terms that overlap it.
std::vector<Tf2Box> disjoint_cover (const std::vector<Tf2Box> &in, const FusedParams &p)
{
  std::vector<Tf2Box> out;
  if (in.empty ())
    return out;
  std::vector<int> cut[3];
  for (const Tf2Box &b : in)
    for (int a = 0; a < 3; ++a)
    {
      cut[a].push_back (b.lo[a]);
      cut[a].push_back (b.hi[a]);
    }
  for (int a = 0; a < 3; ++a)
  {
    std::sort (cut[a].begin (), cut[a].end ());
    cut[a].erase (std::unique (cut[a].begin (), cut[a].end ()), cut[a].end ());
  }
  auto covered = [&] (size_t i, size_t j, size_t l) {
    for (const Tf2Box &b : in)
      if (cut[0][i] >= b.lo[0] && cut[0][i + 1] <= b.hi[0] && cut[1][j] >= b.lo[1] && cut[1][j + 1] <= b.hi[1] &&
          cut[2][l] >= b.lo[2] && cut[2][l + 1] <= b.hi[2])
        return true;
    return false;
  };
  // terms of each component that reach the box at all (bit 4k + t); a
  // cell of the box still tests its own position against them
  auto mask_of = [&] (size_t i, size_t j, size_t l, size_t e) {
    unsigned m = 0;
    for (int k = 0; k < 6; ++k)
      for (int t = 0; t < p.comp[k].nterms; ++t)
      {
        const TermDev &tm = p.comp[k].term[t];
        if (cut[0][i] < tm.hi[0] && cut[0][i + 1] > tm.lo[0] && cut[1][j] < tm.hi[1] && cut[1][j + 1] > tm.lo[1] &&
            cut[2][l] < tm.hi[2] && cut[2][e] > tm.lo[2])
          m |= 1u << (4 * k + t);
      }
    return m;
  };
  for (size_t i = 0; i + 1 < cut[0].size (); ++i)
    for (size_t j = 0; j + 1 < cut[1].size (); ++j)
    {
      size_t l = 0;
      while (l + 1 < cut[2].size ())
      {
        if (!covered (i, j, l))
        {
          ++l;
          continue;
        }
        size_t e = l + 1;
        while (e + 1 < cut[2].size () && covered (i, j, e))
          ++e;
        const unsigned m = mask_of (i, j, l, e);
        Tf2Box b;
        b.lo[0] = cut[0][i];
        b.hi[0] = cut[0][i + 1];
        b.lo[1] = cut[1][j];
        b.hi[1] = cut[1][j + 1];
        b.lo[2] = cut[2][l];
        b.hi[2] = cut[2][e];
        b.mask = m;
        out.push_back (b);
        l = e;
      }
    }
  return out;
}

}  // namespace

std::string tfsf2_regions (const FusedParams &p, std::vector<Tf2Box> r[4])
{
  std::vector<Tf2Box> g[4];
  for (int k = 0; k < 6; ++k)
    for (int t = 0; t < p.comp[k].nterms; ++t)
    {
      const TermDev &tm = p.comp[k].term[t];
      if (tm.lo[0] >= tm.hi[0] || tm.lo[1] >= tm.hi[1] || tm.lo[2] >= tm.hi[2])
        continue;
      // a term box (E or H) grown per axis by (below, above):
      //   T_E: E (0, 0);  R_H1: E (1, 0), H (0, 0);
      //   R_E: E (1, 1), H (0, 1);  R_H2: E (2, 1), H (1, 1)
      const bool e = k < 3;
      const int grow[4][2] = {{0, 0}, {e ? 1 : 0, 0}, {e ? 1 : 0, 1}, {e ? 2 : 1, 1}};
      for (int q = 0; q < 4; ++q)
      {
        if (q == 0 && !e)
          continue;
        Tf2Box b;
        for (int ax = 0; ax < 3; ++ax)
        {
          b.lo[ax] = tm.lo[ax] - grow[q][0];
          b.hi[ax] = tm.hi[ax] + grow[q][1];
        }
        b.mask = 0;
        g[q].push_back (b);
      }
    }
  for (int q = 0; q < 4; ++q)
    r[q] = disjoint_cover (g[q], p);
  // every cell of the regions and its neighbours takes the plain update:
  // inside 2 .. n - 3 and outside every component's PML
  for (int q = 0; q < 4; ++q)
    for (const Tf2Box &b : r[q])
      for (int a = 0; a < 3; ++a)
      {
        if (b.lo[a] < 2 || b.hi[a] > p.g.n[a] - 2)
          return "the TF/SF corrections reach the grid's faces";
        if (p.use_pml)
          for (int k = 0; k < 6; ++k)
            if (b.lo[a] - 1 < p.ilo[k][a] || b.hi[a] + 1 > p.ihi[k][a])
              return "the TF/SF corrections reach into the PML";
      }
  return "";
}

// shared memory of a tile at most: four CTAs per SM (measured at 512^3:
// the step 1.1 % faster than with three CTAs of larger tiles, 2 % faster
// than with two; five or six CTAs spill registers and are slower)
constexpr unsigned kTileSmem = 54u * 1024u;

std::string tfsf2_tiles (const FusedParams &p, const std::vector<Tf2Box> r[4], std::vector<Tf2Tile> &tiles,
                         unsigned &smem)
{
  // the last support's boxes merged where two meet face to face with the
  // same extent across (the cover cuts the thin slabs at every term box edge)
  std::vector<Tf2Box> own = r[3];
  for (bool merged = true; merged;)
  {
    merged = false;
    for (size_t i = 0; i < own.size () && !merged; ++i)
      for (size_t j = 0; j < own.size () && !merged; ++j)
      {
        if (i == j)
          continue;
        for (int a = 0; a < 3 && !merged; ++a)
        {
          const int b = (a + 1) % 3, c = (a + 2) % 3;
          if (own[i].hi[a] == own[j].lo[a] && own[i].lo[b] == own[j].lo[b] && own[i].hi[b] == own[j].hi[b] &&
              own[i].lo[c] == own[j].lo[c] && own[i].hi[c] == own[j].hi[c])
          {
            own[i].hi[a] = own[j].hi[a];
            own.erase (own.begin () + (long) j);
            merged = true;
          }
        }
      }
  }
  tiles.clear ();
  smem = 0;
  for (const Tf2Box &b : own)
  {
    int ext[3], cnt[3];
    for (int a = 0; a < 3; ++a)
      ext[a] = b.hi[a] - b.lo[a];
    // tile extents: up to 8 x 8 x 32 cells, or 16 x 16 across a box that is
    // thin in z (a z face of the TF/SF box), shrunk until a tile's shared
    // memory fits four CTAs per SM; boxes split evenly
    const bool zthin = ext[2] <= 8;
    int cap[3] = {zthin ? 16 : 8, zthin ? 16 : 8, 32};
    for (;;)
    {
      unsigned nE = 1, nH = 1, nP = 1;
      int big = 0;
      for (int a = 0; a < 3; ++a)
      {
        const int d = std::min (ext[a], cap[a]);
        nE *= (unsigned) (d + 3);
        nH *= (unsigned) (d + 2);
        nP *= (unsigned) (d + 4);
        if (d > std::min (ext[big], cap[big]))
          big = a;
      }
      if ((3u * (nE + nH) + nP) * sizeof (float) <= kTileSmem || std::min (ext[big], cap[big]) <= 2)
        break;
      cap[big] = std::min (ext[big], cap[big]) - 1;
    }
    for (int a = 0; a < 3; ++a)
      cnt[a] = (ext[a] + cap[a] - 1) / cap[a];
    for (int i = 0; i < cnt[0]; ++i)
      for (int j = 0; j < cnt[1]; ++j)
        for (int l = 0; l < cnt[2]; ++l)
        {
          Tf2Tile t;
          const int idx[3] = {i, j, l};
          for (int a = 0; a < 3; ++a)
          {
            t.lo[a] = b.lo[a] + ext[a] * idx[a] / cnt[a];
            t.hi[a] = b.lo[a] + ext[a] * (idx[a] + 1) / cnt[a];
          }
          // the terms that reach the tile's E domain [lo - 1, hi + 2) (E
          // components) or its H domain [lo - 1, hi + 1) (H components)
          t.mask = 0;
          for (int k = 0; k < 6; ++k)
            for (int q = 0; q < p.comp[k].nterms; ++q)
            {
              const TermDev &tm = p.comp[k].term[q];
              bool hit = true;
              for (int a = 0; a < 3; ++a)
                hit = hit && tm.lo[a] < t.hi[a] + (k < 3 ? 2 : 1) && tm.hi[a] > t.lo[a] - 1;
              if (hit)
                t.mask |= 1u << (4 * k + q);
            }
          // phase boxes: the supports of dE1, dH1 and dE2 within the phase
          // domains D_E = [lo - 1, hi + 2), D_H = [lo - 1, hi + 1) and
          // U = [lo, hi + 1), relative to lo - 1
          for (int f = 0; f < 3; ++f)
          {
            int d0[3], d1[3], bl[3], bh[3];
            for (int a = 0; a < 3; ++a)
            {
              d0[a] = f == 2 ? t.lo[a] : t.lo[a] - 1;
              d1[a] = f == 1 ? t.hi[a] + 1 : t.hi[a] + (f == 0 ? 2 : 1);
              bl[a] = 1 << 30;
              bh[a] = -(1 << 30);
            }
            for (const Tf2Box &s : r[f])
            {
              int lo[3], hi[3];
              bool ok = true;
              for (int a = 0; a < 3; ++a)
              {
                lo[a] = std::max (s.lo[a], d0[a]);
                hi[a] = std::min (s.hi[a], d1[a]);
                ok = ok && lo[a] < hi[a];
              }
              if (!ok)
                continue;
              for (int a = 0; a < 3; ++a)
              {
                bl[a] = std::min (bl[a], lo[a]);
                bh[a] = std::max (bh[a], hi[a]);
              }
            }
            for (int a = 0; a < 3; ++a)
            {
              const bool empty = bl[a] >= bh[a];
              t.ph[f][a] = (short) (empty ? 0 : bl[a] - (t.lo[a] - 1));
              t.ph[f][3 + a] = (short) (empty ? 0 : bh[a] - (t.lo[a] - 1));
            }
          }
          unsigned nE = 1, nH = 1, nP = 1;
          for (int a = 0; a < 3; ++a)
          {
            nE *= (unsigned) (t.hi[a] - t.lo[a] + 3);
            nH *= (unsigned) (t.hi[a] - t.lo[a] + 2);
            nP *= (unsigned) (t.hi[a] - t.lo[a] + 4);
          }
          smem = std::max (smem, (3u * (nE + nH) + nP) * (unsigned) sizeof (float));
          tiles.push_back (t);
        }
  }
  if (smem > 200u * 1024u)
    return "TF/SF tile too large";
  return "";
}

int launch_tfsf2 (const Tf2Pass &pass, const FusedParams &p, const double *inc_h1, const double *inc_e1,
                  const double *inc_h2, const double *inc_e2, int *err, cudaStream_t s)
{
  if (pass.ntiles <= 0)
    return 0;
  if (p.fp16)
    tfsf2_fused<__half><<<pass.ntiles, 256, pass.smem, s>>> (p, pass.tiles, inc_h1, inc_e1, inc_h2, inc_e2, err);
  else
    tfsf2_fused<float><<<pass.ntiles, 256, pass.smem, s>>> (p, pass.tiles, inc_h1, inc_e1, inc_h2, inc_e2, err);
  return 1;
}

std::string tfsf2_configure (unsigned smem)
{
  if (cudaFuncSetAttribute (tfsf2_fused<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem) !=
          cudaSuccess ||
      cudaFuncSetAttribute (tfsf2_fused<__half>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem) !=
          cudaSuccess)
    return "TF/SF kernel shared-memory set-up failed";
  return "";
}

}  // namespace fdtdb
