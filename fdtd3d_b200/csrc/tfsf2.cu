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
// and c - e_a for E), evaluated in four passes over the supports (the term
// boxes grown by up to two cells), each cell evaluating its own terms once.
// Every cell of the supports takes the plain update in both steps (no PML,
// no point source), which the host checks.
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

// TF/SF change of the curl of component k at (x, y, z) (the single-step
// kernels' tfsf_curl): each term whose box holds the cell subtracts the
// incident value from one neighbour of the curl (n1 - n0) - (n3 - n2).
__device__ __forceinline__ float term_curl (const FusedParams &p, int k, const double *inc, int *err, int x, int y,
                                            int z)
{
  const CompDev &c = p.comp[k];
  float d = 0.f;
  for (int t = 0; t < c.nterms; ++t)
  {
    const TermDev &tm = c.term[t];
    if (x >= tm.lo[0] && x < tm.hi[0] && y >= tm.lo[1] && y < tm.hi[1] && z >= tm.lo[2] && z < tm.hi[2])
    {
      const double diff = inc_at (p.g, inc, p.inc_len, err, tm.inc_comp, x + tm.aux[0], y + tm.aux[1],
                                  z + tm.aux[2]);
      const float dv = (float) (diff * tm.negate) * p.inc_scale[tm.inc_comp];
      d += (tm.slot == 0 || tm.slot == 3) ? dv : -dv;
    }
  }
  return d;
}

// 2 / (eps + eps') of E component k at cell index c (1 without eps)
__device__ __forceinline__ float inv_m (const FusedParams &p, int k, size_t c, size_t sx, int nz)
{
  if (!p.eps)
    return 1.f;
  const size_t st = k == 0 ? sx : (k == 1 ? (size_t) nz : 1);
  return __fdividef (2.f, p.eps[c] + p.eps[c + st]);
}

__device__ __forceinline__ bool box_cell (const Tf2Box &b, int first, int &x, int &y, int &z)
{
  const unsigned ez = (unsigned) (b.hi[2] - b.lo[2]), ey = (unsigned) (b.hi[1] - b.lo[1]);
  const unsigned n = ez * ey * (unsigned) (b.hi[0] - b.lo[0]);
  const unsigned r = (unsigned) first + threadIdx.x;
  if (r >= n)
    return false;
  const unsigned q = r / ez;
  z = b.lo[2] + (int) (r - q * ez);
  y = b.lo[1] + (int) (q % ey);
  x = b.lo[0] + (int) (q / ey);
  return true;
}

// The four passes over their regions (one cell per thread; every cell
// evaluates its own TF/SF terms once):
//   A over R_E: dE1 = S im dE(t1)                          -> sE (0 off the terms)
//   B over R_H1: dH1 = S (curlH sE + dH(t1))               -> sH
//   C over R_E: dE2 = sE + S im (curlE sH + dE(t2))        -> sE, E_new += dE2
//   D over R_H2: dH2 = sH + S (curlH sE + dH(t2))          -> H_new += dH2
// R_E holds the support of dE1 and dE2, R_H1 that of dH1, R_H2 that of dH2.
// sE and sH are zero outside R_E and R_H1 (never written there).
template <typename T, int PASS>
__global__ void __launch_bounds__ (256) tfsf2_pass (const __grid_constant__ FusedParams p, const Tf2Pass pass,
                                                    const double *inc, int *err)
{
  const int r = PASS == 1 ? 1 : (PASS == 3 ? 2 : 0);   // region: 0 R_E, 1 R_H1, 2 R_H2
  const int2 bk = pass.blk[r][blockIdx.x];
  int x, y, z;
  if (!box_cell (pass.boxes[r][bk.x], bk.y, x, y, z))
    return;
  const int ny = p.g.n[1], nz = p.g.n[2];
  const size_t sx = (size_t) ny * nz, sy = nz;
  const float S = p.courant;
  float *const *sE = pass.scratch;
  float *const *sH = pass.scratch + 3;
  const size_t id = (size_t) x * sx + (size_t) y * sy + z;
  if (PASS == 0 || PASS == 2)
  {
    float cu[3];
    if (PASS == 2)
    {
      cu[0] = (sH[2][id] - sH[2][id - sy]) - (sH[1][id] - sH[1][id - 1]);
      cu[1] = (sH[0][id] - sH[0][id - 1]) - (sH[2][id] - sH[2][id - sx]);
      cu[2] = (sH[1][id] - sH[1][id - sx]) - (sH[0][id] - sH[0][id - sy]);
    }
#pragma unroll
    for (int k = 0; k < 3; ++k)
    {
      const float d = (PASS == 2 ? cu[k] : 0.f) + term_curl (p, k, inc, err, x, y, z);
      const float v = d == 0.f ? 0.f : (S * inv_m (p, k, id, sx, nz)) * d;
      if (PASS == 0)
        sE[k][id] = v;
      else
      {
        const float e2 = sE[k][id] + v;
        sE[k][id] = e2;
        if (e2 != 0.f)
        {
          T *f = reinterpret_cast<T *> (p.e_new[k]);
          stf (f, id, ldf (f, id) + e2);
        }
      }
    }
  }
  else
  {
    // curlH of sE (dE1 in pass B, dE2 in pass D)
    const float ex = sE[0][id], ey = sE[1][id], ez = sE[2][id];
    const float a[3] = {(sE[1][id + 1] - ey) - (sE[2][id + sy] - ez), (sE[2][id + sx] - ez) - (sE[0][id + 1] - ex),
                        (sE[0][id + sy] - ex) - (sE[1][id + sx] - ey)};
#pragma unroll
    for (int m = 0; m < 3; ++m)
    {
      const float dh = S * (a[m] + term_curl (p, 3 + m, inc, err, x, y, z));
      if (PASS == 1)
        sH[m][id] = dh;
      else
      {
        const float h2 = sH[m][id] + dh;
        if (h2 != 0.f)
        {
          T *f = reinterpret_cast<T *> (p.h_new[m]);
          stf (f, id, ldf (f, id) + h2);
        }
      }
    }
  }
}

// Disjoint cover of a union of boxes: coordinate compression (every box
// edge is a cut), the covered elementary boxes, runs along z merged.
std::vector<Tf2Box> disjoint_cover (const std::vector<Tf2Box> &in)
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
        Tf2Box b;
        b.lo[0] = cut[0][i];
        b.hi[0] = cut[0][i + 1];
        b.lo[1] = cut[1][j];
        b.hi[1] = cut[1][j + 1];
        b.lo[2] = cut[2][l];
        b.hi[2] = cut[2][e];
        out.push_back (b);
        l = e;
      }
    }
  return out;
}

}  // namespace

std::string tfsf2_regions (const FusedParams &p, std::vector<Tf2Box> r[3])
{
  std::vector<Tf2Box> g[3];
  for (int k = 0; k < 6; ++k)
    for (int t = 0; t < p.comp[k].nterms; ++t)
    {
      const TermDev &tm = p.comp[k].term[t];
      if (tm.lo[0] >= tm.hi[0] || tm.lo[1] >= tm.hi[1] || tm.lo[2] >= tm.hi[2])
        continue;
      // a term box T (E or H) grown per axis by (below, above):
      //   R_E:  E (1, 1), H (0, 1);  R_H1: E (1, 0), H (0, 0);
      //   R_H2: E (2, 1), H (1, 1)
      const bool e = k < 3;
      const int grow[3][2] = {{e ? 1 : 0, 1}, {e ? 1 : 0, 0}, {e ? 2 : 1, 1}};
      for (int q = 0; q < 3; ++q)
      {
        Tf2Box b;
        for (int ax = 0; ax < 3; ++ax)
        {
          b.lo[ax] = tm.lo[ax] - grow[q][0];
          b.hi[ax] = tm.hi[ax] + grow[q][1];
        }
        g[q].push_back (b);
      }
    }
  for (int q = 0; q < 3; ++q)
    r[q] = disjoint_cover (g[q]);
  // every cell of the regions and its neighbours takes the plain update:
  // inside 2 .. n - 3 and outside every component's PML
  for (int q = 0; q < 3; ++q)
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

std::string tfsf2_blocks (const std::vector<Tf2Box> &boxes, std::vector<int2> &blk)
{
  blk.clear ();
  for (size_t q = 0; q < boxes.size (); ++q)
  {
    const Tf2Box &b = boxes[q];
    const long long cells = (long long) (b.hi[0] - b.lo[0]) * (b.hi[1] - b.lo[1]) * (b.hi[2] - b.lo[2]);
    if (cells >= (1ll << 31))
      return "TF/SF box too large";
    for (long long f = 0; f < cells; f += 256)
      blk.push_back (make_int2 ((int) q, (int) f));
  }
  return "";
}

int launch_tfsf2 (const Tf2Pass &pass, const FusedParams &p, const double *inc_h1, const double *inc_e1,
                  const double *inc_h2, const double *inc_e2, int *err, cudaStream_t s)
{
  if (pass.nblk[0] <= 0)
    return 0;
  if (p.fp16)
  {
    tfsf2_pass<__half, 0><<<pass.nblk[0], 256, 0, s>>> (p, pass, inc_h1, err);
    tfsf2_pass<__half, 1><<<pass.nblk[1], 256, 0, s>>> (p, pass, inc_e1, err);
    tfsf2_pass<__half, 2><<<pass.nblk[0], 256, 0, s>>> (p, pass, inc_h2, err);
    tfsf2_pass<__half, 3><<<pass.nblk[2], 256, 0, s>>> (p, pass, inc_e2, err);
  }
  else
  {
    tfsf2_pass<float, 0><<<pass.nblk[0], 256, 0, s>>> (p, pass, inc_h1, err);
    tfsf2_pass<float, 1><<<pass.nblk[1], 256, 0, s>>> (p, pass, inc_e1, err);
    tfsf2_pass<float, 2><<<pass.nblk[0], 256, 0, s>>> (p, pass, inc_h2, err);
    tfsf2_pass<float, 3><<<pass.nblk[2], 256, 0, s>>> (p, pass, inc_e2, err);
  }
  return 4;
}

}  // namespace fdtdb
