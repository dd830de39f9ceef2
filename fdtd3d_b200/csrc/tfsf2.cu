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
// boxes grown by up to two cells), each cell evaluating the terms that cover
// it (a mask per region box) once.
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

// The same over the terms of `mask` (bit t: term t of component k), those
// that overlap the cell's box.
__device__ __forceinline__ float term_curl_masked (const FusedParams &p, int k, unsigned mask, const double *inc,
                                                   int *err, int x, int y, int z)
{
  const CompDev &c = p.comp[k];
  float d = 0.f;
#pragma unroll
  for (int t = 0; t < kMaxTerms; ++t)
    if ((mask >> t) & 1u)
    {
      const TermDev &tm = c.term[t];
      if (!(x >= tm.lo[0] && x < tm.hi[0] && y >= tm.lo[1] && y < tm.hi[1] && z >= tm.lo[2] && z < tm.hi[2]))
        continue;
      const double diff = inc_at (p.g, inc, p.inc_len, err, tm.inc_comp, x + tm.aux[0], y + tm.aux[1],
                                  z + tm.aux[2]);
      const float dv = (float) (diff * tm.negate) * p.inc_scale[tm.inc_comp];
      d += (tm.slot == 0 || tm.slot == 3) ? dv : -dv;
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
// evaluates only the terms of its box's mask):
//   A over T_E:  dE1 = S im dE(t1)                         -> sE1
//   B over R_H1: dH1 = S (curlH sE1 + dH(t1))              -> sH1
//   C over R_E:  dE2 = sE1 + S im (curlE sH1 + dE(t2))     -> sE2, E_new += dE2
//   D over R_H2: dH2 = sH1 + S (curlH sE2 + dH(t2))        -> H_new += dH2
// T_E holds the E term cells, R_H1 the support of dH1, R_E that of dE1 and
// dE2, R_H2 that of dH2; sE1, sH1 and sE2 are zero outside T_E, R_H1 and R_E
// (never written there).
template <typename T, int PASS>
__global__ void __launch_bounds__ (256) tfsf2_pass (const __grid_constant__ FusedParams p, const Tf2Pass pass,
                                                    const double *inc, int *err)
{
  const int2 bk = pass.blk[PASS][blockIdx.x];
  const Tf2Box &box = pass.boxes[PASS][bk.x];
  int x, y, z;
  if (!box_cell (box, bk.y, x, y, z))
    return;
  const unsigned mask = box.mask;
  const int ny = p.g.n[1], nz = p.g.n[2];
  const size_t sx = (size_t) ny * nz, sy = nz;
  const float S = p.courant;
  float *const *sE1 = pass.scratch;
  float *const *sH1 = pass.scratch + 3;
  float *const *sE2 = pass.scratch + 6;
  const size_t id = (size_t) x * sx + (size_t) y * sy + z;
  if (PASS == 0 || PASS == 2)
  {
    float cu[3] = {0.f, 0.f, 0.f};
    if (PASS == 2)
    {
      cu[0] = (sH1[2][id] - sH1[2][id - sy]) - (sH1[1][id] - sH1[1][id - 1]);
      cu[1] = (sH1[0][id] - sH1[0][id - 1]) - (sH1[2][id] - sH1[2][id - sx]);
      cu[2] = (sH1[1][id] - sH1[1][id - sx]) - (sH1[0][id] - sH1[0][id - sy]);
    }
#pragma unroll
    for (int k = 0; k < 3; ++k)
    {
      const unsigned mk = (mask >> (4 * k)) & 15u;
      const float d = cu[k] + (mk ? term_curl_masked (p, k, mk, inc, err, x, y, z) : 0.f);
      const float v = d == 0.f ? 0.f : (S * inv_m (p, k, id, sx, nz)) * d;
      if (PASS == 0)
        sE1[k][id] = v;
      else
      {
        const float e2 = sE1[k][id] + v;
        sE2[k][id] = e2;
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
    // curlH of the E corrections (dE1 in pass B, dE2 in pass D)
    float *const *sE = PASS == 1 ? sE1 : sE2;
    const float ex = sE[0][id], ey = sE[1][id], ez = sE[2][id];
    const float a[3] = {(sE[1][id + 1] - ey) - (sE[2][id + sy] - ez), (sE[2][id + sx] - ez) - (sE[0][id + 1] - ex),
                        (sE[0][id + sy] - ex) - (sE[1][id + sx] - ey)};
#pragma unroll
    for (int m = 0; m < 3; ++m)
    {
      const unsigned mk = (mask >> (4 * (3 + m))) & 15u;
      const float dh = S * (a[m] + (mk ? term_curl_masked (p, 3 + m, mk, inc, err, x, y, z) : 0.f));
      if (PASS == 1)
        sH1[m][id] = dh;
      else
      {
        const float h2 = sH1[m][id] + dh;
        if (h2 != 0.f)
        {
          T *f = reinterpret_cast<T *> (p.h_new[m]);
          stf (f, id, ldf (f, id) + h2);
        }
      }
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
  if (pass.nblk[2] <= 0)
    return 0;
  int n = 0;
  auto go = [&] (auto kern, int q, const double *inc) {
    if (pass.nblk[q] > 0)
    {
      kern<<<pass.nblk[q], 256, 0, s>>> (p, pass, inc, err);
      ++n;
    }
  };
  if (p.fp16)
  {
    go (tfsf2_pass<__half, 0>, 0, inc_h1);
    go (tfsf2_pass<__half, 1>, 1, inc_e1);
    go (tfsf2_pass<__half, 2>, 2, inc_h2);
    go (tfsf2_pass<__half, 3>, 3, inc_e2);
  }
  else
  {
    go (tfsf2_pass<float, 0>, 0, inc_h1);
    go (tfsf2_pass<float, 1>, 1, inc_e1);
    go (tfsf2_pass<float, 2>, 2, inc_h2);
    go (tfsf2_pass<float, 3>, 3, inc_e2);
  }
  return n;
}

}  // namespace fdtdb
