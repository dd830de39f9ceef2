// sweep3d.cu - TMA-pipelined one-sweep E+H leapfrog step (3-D, FP32 and
// FP16-storage forms).
//
// Same arithmetic and double-buffered data flow as fused3d.cu (every value
// is read from the old buffers and written to the new ones once per step),
// reorganised for the B200 memory system:
//
//  * A CTA owns a tile of 128 z cells x (WY - 1) y rows and marches x over a
//    chunk of planes.  Lane l of warp w handles the four cells
//    z0 + 4l .. z0 + 4l + 3 of row y0 + w, so every global access is a
//    16-byte vector per lane.  Warp WY - 1 is the y ring: it recomputes E on
//    the row after the tile (needed by H of the last owned row) and stores
//    nothing; lane 31 recomputes E on the z ring cell z0 + 128.
//  * Per plane x, one elected thread streams H(x) (with the y - 1 row and a
//    16-byte z halo on both sides), E_old(x), eps(x), eps(x + 1) and, on
//    planes that hold PML cells, the PML auxiliaries into shared memory with
//    cp.async.bulk.tensor, three stages deep, completion signalled on an
//    mbarrier (bounded waits).  Neighbour values then come from shared
//    memory, so the compute is plain vector arithmetic with no global-memory
//    latency on its critical path.
//  * E_new(x) goes to global memory and to a three-deep shared exchange
//    buffer; H_new(x - 1) reads E_new(x - 1) (with its y + 1 / z + 1
//    neighbours) from there and E_new(x) from registers.  One __syncthreads
//    per plane orders everything.
//  * CTAs are persistent and take (z tile, y tile, x chunk) items from an
//    atomic counter, so tiles with PML or TF/SF work balance out.
// PML auxiliaries, TF/SF corrections and the point source are applied only
// on the lanes whose cells need them.
#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <mutex>
#include <type_traits>
#include <vector>

#include "incident_dev.cuh"
#include "sweep3d.h"
#include "tma.cuh"

namespace fdtdb {

namespace {

using tma::global_ns;
using tma::mbar_expect_tx;
using tma::mbar_init;
using tma::mbar_wait;
using tma::smem_addr;

__device__ __forceinline__ void tma_load_3d (uint32_t dst, const CUtensorMap *map, int c0, int c1, int c2,
                                             uint32_t bar)
{
  tma::load_3d (dst, map, c0, c1, c2, bar);
}

constexpr int TZ = 128;           // z cells per tile: 32 lanes x 4
constexpr int PW = TZ + 4;        // eps / auxiliary / exchange row width in floats (z0 .. z0 + 131)
constexpr int NST = 3;            // pipeline stages (plane index mod 3 = stage = exchange buffer)
constexpr int MAXC = 64;          // largest x chunk when PML coefficient tables are staged

template <typename T, int WY>
struct Smem
{
  static constexpr int HZ = 16 / (int) sizeof (T);   // z halo: one 16-byte unit
  static constexpr int HW = TZ + 2 * HZ;             // H row: z0 - HZ .. z0 + TZ + HZ - 1
  static constexpr int EW = TZ + HZ;                 // E row: z0 .. z0 + TZ + HZ - 1
  static constexpr int AN = 32;                      // narrow auxiliary box width (floats)
  static constexpr int XW = MAXC + 2;                // x-table entries per item (planes xa - 1 .. xb + 1)
  static constexpr unsigned rnd (unsigned b) { return (b + 127u) / 128u * 128u; }
  static constexpr unsigned H_B = rnd (sizeof (T) * HW * (WY + 1));
  static constexpr unsigned E_B = rnd (sizeof (T) * EW * WY);
  static constexpr unsigned P_B = rnd (sizeof (float) * PW * WY);   // one eps / auxiliary / exchange plane
  // stage: H x3, E x3, eps(x), eps(x + 1), auxiliaries of Ex..Ez at x and Hx..Hz at x - 1
  static constexpr unsigned OFF_E = 3 * H_B;
  static constexpr unsigned OFF_P = OFF_E + 3 * E_B;
  static constexpr unsigned OFF_A = OFF_P + 2 * P_B;
  static constexpr unsigned STAGE = OFF_A + 6 * P_B;
  static constexpr unsigned OFF_N = NST * STAGE;     // exchange: [3 buffers][Ex, Ez] rows
  // PML coefficient pairs of the item: along z [6][2][PW], y [6][2][WY], x [6][2][XW]
  static constexpr unsigned OFF_T = OFF_N + 6 * P_B;
  static constexpr int TY0 = 6 * 2 * PW;
  static constexpr int TX0 = TY0 + 6 * 2 * WY;
  static constexpr unsigned T_B = rnd (sizeof (float) * (TX0 + 6 * 2 * XW));
  static constexpr unsigned OFF_BAR = OFF_T + T_B;
  static constexpr unsigned TOTAL = OFF_BAR + 128 + 128;   // + room to align the base to 128 bytes
  // bytes each group of copies delivers (full boxes, halo and fill included)
  static constexpr unsigned TX_HE = 3u * sizeof (T) * HW * (WY + 1) + 3u * sizeof (T) * EW * WY;
  static constexpr unsigned TX_P = 2u * sizeof (float) * PW * WY;
  static constexpr unsigned TX_A = 6u * sizeof (float) * PW * WY;
  static constexpr unsigned TX_AN = 6u * sizeof (float) * AN * WY;
  static constexpr unsigned TX_AN4 = 4u * sizeof (float) * AN * WY;   // z-edge items: no Ex / Hx auxiliary
};

// ------------------------------------------------------- element conversions

template <typename T>
struct Vec;

template <>
struct Vec<float>
{
  static __device__ __forceinline__ void ld4 (const float *s, float v[4])
  {
    const float4 t = *reinterpret_cast<const float4 *> (s);
    v[0] = t.x;
    v[1] = t.y;
    v[2] = t.z;
    v[3] = t.w;
  }
  static __device__ __forceinline__ float ld1 (const float *s) { return *s; }
  // streaming (evict-first) store: the new buffers are read again only in
  // the next step, after far more than L2 holds has passed through it
  static __device__ __forceinline__ void st4 (float *g, const float v[4])
  {
    __stcs (reinterpret_cast<float4 *> (g), make_float4 (v[0], v[1], v[2], v[3]));
  }
};

template <>
struct Vec<__half>
{
  static __device__ __forceinline__ void ld4 (const __half *s, float v[4])
  {
    const uint2 t = *reinterpret_cast<const uint2 *> (s);
    const float2 a = __half22float2 (*reinterpret_cast<const __half2 *> (&t.x));
    const float2 b = __half22float2 (*reinterpret_cast<const __half2 *> (&t.y));
    v[0] = a.x;
    v[1] = a.y;
    v[2] = b.x;
    v[3] = b.y;
  }
  static __device__ __forceinline__ float ld1 (const __half *s) { return __half2float (*s); }
  static __device__ __forceinline__ void st4 (__half *g, const float v[4])
  {
    __half2 a = __floats2half2_rn (v[0], v[1]);
    __half2 b = __floats2half2_rn (v[2], v[3]);
    uint2 t;
    t.x = *reinterpret_cast<unsigned *> (&a);
    t.y = *reinterpret_cast<unsigned *> (&b);
    __stcs (reinterpret_cast<uint2 *> (g), t);
  }
};

__device__ __forceinline__ void lds4f (const float *s, float v[4])
{
  Vec<float>::ld4 (s, v);
}

__device__ __forceinline__ void sts4f (float *s, const float v[4])
{
  *reinterpret_cast<float4 *> (s) = make_float4 (v[0], v[1], v[2], v[3]);
}

// ------------------------------------------------------------ cell physics

__device__ __forceinline__ bool on_face (const int *planes, int v)
{
  return v == planes[0] || v == planes[1] || v == planes[2] || v == planes[3];
}

// TF/SF change of the curl of component k at (x, y, z).  Each matching term
// subtracts the incident value from one neighbour of the curl
// (n1 - n0) - (n3 - n2): slots 0 and 3 raise the curl by that value, slots
// 1 and 2 lower it (InternalScheme.inc.h:1386-1835).
__device__ __forceinline__ float tfsf_curl (const FusedParams &p, int k, const double *inc, int *err, int x, int y,
                                            int z)
{
  const CompDev &c = p.comp[k];
  float d = 0.f;
  for (int t = 0; t < c.nterms; ++t)
  {
    const TermDev &tm = c.term[t];
    if (x >= tm.lo[0] && x < tm.hi[0] && y >= tm.lo[1] && y < tm.hi[1] && z >= tm.lo[2] && z < tm.hi[2])
    {
      const double diff =
          inc_at (p.g, inc, p.inc_len, err, tm.inc_comp, x + tm.aux[0], y + tm.aux[1], z + tm.aux[2]);
      const float dv = (float) (diff * tm.negate) * p.inc_scale[tm.inc_comp];
      d += (tm.slot == 0 || tm.slot == 3) ? dv : -dv;
    }
  }
  return d;
}

// Out-of-line TF/SF curl change for the sweep's rarely taken in-kernel path
// (TF/SF bands that reach the PML), so that its code stays out of the hot
// loop body.
__device__ __noinline__ float tfsf_curl_cold (const FusedParams *p, int k, const double *inc, int *err, int x, int y,
                                              int z)
{
  return tfsf_curl (*p, k, inc, err, x, y, z);
}

// Pair of PML coefficient tables of component k that runs along an axis:
// pair 0 (ca1, sq1) runs along axis k + 1, pair 1 (p5, q5) along k + 2,
// pair 2 (g4p, g4m) along k itself (the reference's sigma choice per
// component, InternalScheme.inc.h:2551-2640).
__host__ __device__ constexpr int pair_along (int k, int axis)
{
  return (k + 1) % 3 == axis ? 0 : ((k + 2) % 3 == axis ? 1 : 2);
}

// The item's PML coefficient pairs staged in shared memory, per component k
// and pair element t: z[(2k + t) * PW + column], y[(2k + t) * WY + row],
// x[(2k + t) * (MAXC + 2) + plane - (xa - 1)].
struct PmlTabs
{
  const float *z, *y, *x;
};

// PML update of component K on the cells of mask pm among a lane's four
// cells: X_new = ca1 X + sq1 curl, F = p5 F + (g4p X_new - g4m X) q5 / m.
// Branch-free over the cells; cells outside pm keep fn and their X.
template <int K, int WY>
__device__ __forceinline__ void pml_vec (const PmlTabs &t, float S, int row, int plane, int col, unsigned pm,
                                         const float xo[4], const float cu[4], const float im[4], const float fo[4],
                                         float fn[4], float xn[4])
{
  constexpr int pz = pair_along (K, 2), py = pair_along (K, 1), px = pair_along (K, 0);
  constexpr int XW = MAXC + 2;
  float c[3][2][4];
#pragma unroll
  for (int e = 0; e < 2; ++e)
  {
    lds4f (t.z + (2 * K + e) * PW + col, c[pz][e]);
    const float vy = t.y[(2 * K + e) * WY + row];
    const float vx = t.x[(2 * K + e) * XW + plane];
#pragma unroll
    for (int j = 0; j < 4; ++j)
    {
      c[py][e][j] = vy;
      c[px][e][j] = vx;
    }
  }
#pragma unroll
  for (int j = 0; j < 4; ++j)
  {
    const float n = c[0][0][j] * xo[j] + c[0][1][j] * cu[j];
    const float f = c[1][0][j] * fo[j] + (c[2][0][j] * n - c[2][1][j] * xo[j]) * c[1][1][j] * im[j];
    const bool on = (pm >> j) & 1u;
    fn[j] = on ? f : fn[j];
    xn[j] = on ? n : xo[j];
  }
}

// The same for one cell (the z ring cell, column 128 of the tile).
template <int K, int WY>
__device__ __forceinline__ float pml_one (const PmlTabs &t, float S, int row, int plane, int col, float xo, float cu,
                                          float im, float fo)
{
  constexpr int pz = pair_along (K, 2), py = pair_along (K, 1);
  constexpr int XW = MAXC + 2;
  float c[3][2];
#pragma unroll
  for (int e = 0; e < 2; ++e)
#pragma unroll
    for (int q = 0; q < 3; ++q)
      c[q][e] = q == pz ? t.z[(2 * K + e) * PW + col]
                        : (q == py ? t.y[(2 * K + e) * WY + row] : t.x[(2 * K + e) * XW + plane]);
  const float n = c[0][0] * xo + c[0][1] * cu;
  return c[1][0] * fo + (c[2][0] * n - c[2][1] * xo) * c[1][1] * im;
}

// z-edge items (x and y interior): only the z pair of each component
// differs from the sigma = 0 identity, and the item's z tables hold it in
// the form of one branch-free update for PML and interior cells alike:
//   (p5, q5) along z (Ex, Hx) as (p5, S q5): F = p5 F + S q5 im curl; the
//     auxiliary cancels, since ca1 = 1, sq1 = S, g4p = g4m = 1 make
//     X_new - X = S curl, so none is kept;
//   (ca1, sq1) along z (Ey, Hy) as (ca1 - 1, sq1):
//     X_new = ca1 X + sq1 curl, F = F + ((ca1 - 1) X + sq1 curl) im;
//   (g4p, g4m) along z (Ez, Hz) as (S g4p, g4p - g4m):
//     X_new = X + S curl, F = F + ((g4p - g4m) X + S g4p curl) im.
// With the identity values each form is exactly the lean update
// F + (S im) curl, so interior cells match the lean class bit for bit; X is
// taken as 0 on cells that are not PML cells of the component.
__host__ __device__ inline void zedge_pair (int k, float a, float b, float S, float &c0, float &c1)
{
  switch (pair_along (k, 2))
  {
    case 1: c0 = a; c1 = S * b; break;
    case 0: c0 = a - 1.f; c1 = b; break;
    default: c0 = S * a; c1 = a - b; break;
  }
}

// Component K on a lane's four cells of a z-edge item; xn gets X_new on the
// cells of pm (0 elsewhere) for the two components that keep an auxiliary.
template <int K>
__device__ __forceinline__ void zedge_vec (const float *tz, int col, float S, unsigned upd, unsigned pm,
                                           const float xo[4], const float cu[4], const float im[4],
                                           const float fo[4], float fn[4], float xn[4])
{
  constexpr int pz = pair_along (K, 2);
  float c0[4], c1[4];
  lds4f (tz + (2 * K) * PW + col, c0);
  lds4f (tz + (2 * K + 1) * PW + col, c1);
#pragma unroll
  for (int j = 0; j < 4; ++j)
  {
    const bool on = (pm >> j) & 1u;
    const float x = on ? xo[j] : 0.f;
    float f;
    if (pz == 1)
      f = fmaf (im[j] * c1[j], cu[j], c0[j] * fo[j]);
    else if (pz == 0)
    {
      f = fmaf (c1[j] * im[j], cu[j], fmaf (c0[j] * im[j], x, fo[j]));
      xn[j] = on ? fmaf (c0[j], x, fmaf (c1[j], cu[j], x)) : 0.f;
    }
    else
    {
      f = fmaf (c0[j] * im[j], cu[j], fmaf (c1[j] * im[j], x, fo[j]));
      xn[j] = on ? fmaf (S, cu[j], x) : 0.f;
    }
    fn[j] = ((upd >> j) & 1u) ? f : fo[j];
  }
}

// ------------------------------------------------------------ item classes

// Class of work item `item` (the kernel instantiation that runs it):
//   2 (full): TF/SF corrections inside the sweep, or a point source on a
//     plane the item updates (E on x = xa .. xb + 1, H on x = xa .. xb);
//   3 (PML): otherwise, a PML cell of any component off the z edges of the
//     tile (full-width auxiliary boxes on every plane);
//   1 (z edge): PML cells only in z columns that one narrow window of the
//     tile holds (the ring column included), x and y interior;
//   0 (lean): none of these.
// Shared by the host (launch and counts) and the kernels (item pick).
__host__ __device__ inline int sweep_item_class (const FusedParams &p, const SweepWork &wk, int wy, int item,
                                                 bool tfsf_in)
{
  const int nx = p.g.n[0], ny = p.g.n[1], nz = p.g.n[2];
  const int zt = item % wk.nzt;
  const int yt = (item / wk.nzt) % wk.nyt;
  const int ch = item / (wk.nzt * wk.nyt);
  const int z0 = zt * TZ, y0 = 1 + yt * (wy - 1), xa = wk.xcut[ch];
  const int xb = wk.xcut[ch + 1] - 1;
  if (tfsf_in || !wk.lean)
    return 2;
  if (p.ps_mask && p.ps[0] >= xa && p.ps[0] <= xb + 1)
    return 2;
  if (!p.use_pml)
    return 0;
  const int yhi = y0 + wy - 1 < ny - 2 ? y0 + wy - 1 : ny - 2;
  // x and y must be interior for every component
  for (int k = 0; k < 6; ++k)
  {
    const int xhi = k < 3 ? (xb + 1 < nx - 2 ? xb + 1 : nx - 2) : xb;
    if (xa < p.ilo[k][0] || xhi >= p.ihi[k][0] || y0 < p.ilo[k][1] || yhi >= p.ihi[k][1])
      return 3;
  }
  // z: updated columns cmin .. cmax of the tile against the common interior
  int zin_lo = 0, zin_hi = nz;
  for (int k = 0; k < 6; ++k)
  {
    zin_lo = p.ilo[k][2] > zin_lo ? p.ilo[k][2] : zin_lo;
    zin_hi = p.ihi[k][2] < zin_hi ? p.ihi[k][2] : zin_hi;
  }
  const int cmin = 1 - z0 > 0 ? 1 - z0 : 0;
  const int cmax = nz - 2 - z0 < TZ ? nz - 2 - z0 : TZ;
  const int lo_end = zin_lo - z0 < cmax + 1 ? zin_lo - z0 : cmax + 1;
  const int hi_beg = zin_hi - z0 > cmin ? zin_hi - z0 : cmin;
  const bool zlow = lo_end > cmin, zhigh = hi_beg <= cmax;
  if (!zlow && !zhigh)
    return 0;
  if (zlow && zhigh)
    return 3;
  const int az0 = (zlow ? cmin : hi_beg) & ~3;
  const int width = (zlow ? lo_end : cmax + 1) - az0;
  return width <= 32 ? 1 : 3;
}

// ------------------------------------------------------------------ kernel

// MODE (item class, see sweep_item_class): 0 = lean, no PML cell, point
// source or in-sweep TF/SF (straight-line planes); 1 = z edge, PML cells
// only in the z columns of one narrow window; 3 = PML anywhere, full-width
// auxiliary boxes on every plane; 2 = full (in-sweep TF/SF, point sources,
// auxiliary box width chosen per plane).  Classes 0, 1 and 3 unroll the
// plane loop by the stage count (compile-time stage indices).  Each
// instantiation takes only its own items from its own counter.
template <typename T, int WY, int MODE>
__global__ void __launch_bounds__ (32 * WY, 1)
    sweep3d_kernel (const __grid_constant__ SweepMaps maps, const __grid_constant__ FusedParams p,
                    const SweepWork wk, int *err)
{
  using L = Smem<T, WY>;
  constexpr int HZ = L::HZ, HW = L::HW, EW = L::EW, AN = L::AN, XW = L::XW;
  constexpr int HS = L::H_B / sizeof (T), ES = L::E_B / sizeof (T), PS = L::P_B / sizeof (float);
  constexpr unsigned kLanes = 0xffffffffu;   // shuffle mask: the whole warp
  extern __shared__ __align__ (128) unsigned char smem_raw[];
  // grabbed item, double buffered by grab parity: a CTA that skips an item
  // of another class passes only one barrier before its next grab, so the
  // next write must not land in the slot slower warps may still be reading
  __shared__ int s_item[2];
  __shared__ int s_abort[2];   // per plane parity: a copy did not arrive in time

  const int lane = threadIdx.x, w = threadIdx.y;
  const int tid = w * 32 + lane;
  const bool leader = tid == 0;
  const int nx = p.g.n[0], ny = p.g.n[1], nz = p.g.n[2];
  const size_t sx = (size_t) ny * nz;
  // 128-byte aligned base of the dynamic shared memory (TMA destinations)
  const uint32_t raw = smem_addr (smem_raw);
  const uint32_t sbase = (raw + 127u) & ~127u;
  unsigned char *const smem = smem_raw + (sbase - raw);
  const uint32_t bar = sbase + L::OFF_BAR;
  const bool has_eps = p.eps != nullptr;
  const float S = p.courant;
  const float one4[4] = {1.f, 1.f, 1.f, 1.f};
  const bool tfsf_in = p.use_tfsf && !p.tfsf_post;   // corrections inside the sweep
  float *const Tab = reinterpret_cast<float *> (smem + L::OFF_T);
  const PmlTabs tabs{Tab, Tab + L::TY0, Tab + L::TX0};
  // interior z range common to every component (cells outside it are PML for some component)
  int zin_lo = 0, zin_hi = nz;
#pragma unroll
  for (int k = 0; k < 6; ++k)
  {
    zin_lo = max (zin_lo, p.ilo[k][2]);
    zin_hi = min (zin_hi, p.ihi[k][2]);
  }

  if (leader)
  {
#pragma unroll
    for (int st = 0; st < NST; ++st)
      mbar_init (bar + 8 * st, 1);
    asm volatile ("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_abort[0] = s_abort[1] = 0;
  }
  __syncthreads ();

  // Auxiliary mode of plane x of the tile at (z0, y0): 0 = no PML cell of
  // Ex..Ez at x nor of Hx..Hz at x - 1; 1 = PML cells only in the z columns
  // of the narrow window (az0 is its first column, nar_ok whether the
  // tile's z-PML columns fit in one); 2 = full-width auxiliary planes.
  auto aux_mode = [&] (int x, int y0, bool zpml, bool nar_ok) -> int {
    if (!p.use_pml)
      return 0;
    const int yhi = min (y0 + WY - 1, ny - 2);
    bool xyin = true;
#pragma unroll
    for (int k = 0; k < 6; ++k)
    {
      const int xx = k < 3 ? x : x - 1;
      xyin = xyin && xx >= p.ilo[k][0] && xx < p.ihi[k][0] && y0 >= p.ilo[k][1] && yhi < p.ihi[k][1];
    }
    if (xyin && !zpml)
      return 0;
    return (xyin && nar_ok) ? 1 : 2;
  };

  // stage `st` <- plane x of the tile at (z0, y0)
  auto issue = [&] (unsigned st, int x, int z0, int y0, int mode, int az0) {
    const uint32_t s = sbase + st * L::STAGE;
    const uint32_t b = bar + 8 * st;
    mbar_expect_tx (b, L::TX_HE + (has_eps ? L::TX_P : 0u) +
                           (mode == 2 ? L::TX_A : (mode == 1 ? (MODE == 1 ? L::TX_AN4 : L::TX_AN) : 0u)));
#pragma unroll
    for (int c = 0; c < 3; ++c)
      tma_load_3d (s + c * L::H_B, &maps.h[c], z0 - HZ, y0 - 1, x, b);
#pragma unroll
    for (int c = 0; c < 3; ++c)
      tma_load_3d (s + L::OFF_E + c * L::E_B, &maps.e[c], z0, y0, x, b);
    if (has_eps)
    {
      tma_load_3d (s + L::OFF_P, &maps.eps, z0, y0, x, b);
      tma_load_3d (s + L::OFF_P + L::P_B, &maps.eps, z0, y0, min (x + 1, nx - 1), b);
    }
    if (mode)
    {
#pragma unroll
      for (int c = 0; c < 6; ++c)
      {
        if (MODE == 1 && (c == 0 || c == 3))
          continue;
        const int xx = c < 3 ? x : max (x - 1, 0);
        if (mode == 2)
          tma_load_3d (s + L::OFF_A + c * L::P_B, &maps.aux[c], z0, y0, xx, b);
        else
          tma_load_3d (s + L::OFF_A + c * L::P_B, &maps.auxn[c], z0 + az0, y0, xx, b);
      }
    }
  };

  unsigned phase = 0;   // bit s: parity of the next completion of stage s
  bool aborted = false;
  unsigned grab = 0;    // items grabbed by this CTA (selects the s_item slot)
  for (;;)
  {
    if (leader)
    {
      const int idx = (int) atomicAdd (wk.ctr + 2 * MODE, 1ull);
      s_item[grab & 1u] = wk.list ? (idx < wk.nlist ? wk.list[idx] : wk.nitems) : idx;
    }
    __syncthreads ();
    const int item = s_item[grab & 1u];
    ++grab;
    if (item >= wk.nitems)
      break;
    if (sweep_item_class (p, wk, WY, item, tfsf_in) != MODE)
      continue;
    const int zt = item % wk.nzt;
    const int yt = (item / wk.nzt) % wk.nyt;
    const int ch = item / (wk.nzt * wk.nyt);
    const int z0 = zt * TZ;
    const int y0 = 1 + yt * (WY - 1);
    const int xa = wk.xcut[ch];
    const int xb = wk.xcut[ch + 1] - 1;
    const int np = xb - xa + 3;   // planes xa - 1 .. xb + 1 (at least 3)

    // z-PML columns of the tile (ring column included) and whether one
    // narrow window of AN columns holds them
    const int cmin = max (0, 1 - z0), cmax = min (TZ, nz - 2 - z0);
    const int lo_end = min (zin_lo - z0, cmax + 1);    // low-side PML columns [cmin, lo_end)
    const int hi_beg = max (zin_hi - z0, cmin);        // high-side PML columns [hi_beg, cmax]
    const bool zlow = lo_end > cmin, zhigh = hi_beg <= cmax;
    const bool zpml = zlow || zhigh;
    int az0 = 0;
    bool nar_ok = false;
    if (zlow && !zhigh)
    {
      az0 = cmin & ~3;
      nar_ok = lo_end - az0 <= AN;
    }
    else if (zhigh && !zlow)
    {
      az0 = hi_beg & ~3;
      nar_ok = cmax + 1 - az0 <= AN;
    }

    if (leader)
    {
#pragma unroll
      for (int k = 0; k < NST; ++k)
        issue (k, xa - 1 + k, z0, y0,
               MODE == 0 ? 0 : (MODE == 1 ? 1 : (MODE == 3 ? 2 : aux_mode (xa - 1 + k, y0, zpml, nar_ok))), az0);
    }
    // PML coefficient pairs of this item (read after the first plane's barrier)
    if (MODE == 1 && p.use_pml)
    {
      for (int q = tid; q < 6 * PW; q += 32 * WY)
      {
        const int k = q / PW, col = q % PW, z = z0 + col;
        const int pz = pair_along (k, 2);
        float c0 = 0.f, c1 = 0.f;
        if (z < nz)
          zedge_pair (k, __ldg (p.tab[k][2 * pz] + z), __ldg (p.tab[k][2 * pz + 1] + z), S, c0, c1);
        Tab[(2 * k) * PW + col] = c0;
        Tab[(2 * k + 1) * PW + col] = c1;
      }
    }
    else if ((MODE == 2 || MODE == 3) && p.use_pml)
    {
      for (int q = tid; q < 6 * 2 * PW; q += 32 * WY)
      {
        const int k = q / (2 * PW), e = (q / PW) % 2, z = z0 + q % PW;
        Tab[q] = z < nz ? __ldg (p.tab[k][2 * pair_along (k, 2) + e] + z) : 0.f;
      }
      for (int q = tid; q < 6 * 2 * WY; q += 32 * WY)
      {
        const int k = q / (2 * WY), e = (q / WY) % 2, yy = min (y0 + q % WY, ny - 1);
        Tab[L::TY0 + q] = __ldg (p.tab[k][2 * pair_along (k, 1) + e] + yy);
      }
      for (int q = tid; q < 6 * 2 * XW; q += 32 * WY)
      {
        const int k = q / (2 * XW), e = (q / XW) % 2, xx = min (max (xa - 1 + q % XW, 0), nx - 1);
        Tab[L::TX0 + q] = __ldg (p.tab[k][2 * pair_along (k, 0) + e] + xx);
      }
    }

    // ---- per-lane / per-row constants of this item
    const int zl = 4 * lane;
    const int zc = z0 + zl;
    const bool lane_ok = zc < nz;
    const int y = y0 + w;
    const bool yupd = y <= ny - 2;
    const bool own_row = w < WY - 1 && yupd;
    const size_t rowoff = (size_t) y * nz + zc;
    unsigned zupd = 0, zface = 0, zin = 0, yin = 0;   // zin bit 4k + j, yin bit k
#pragma unroll
    for (int j = 0; j < 4; ++j)
    {
      const int z = zc + j;
      if (z >= 1 && z <= nz - 2)
        zupd |= 1u << j;
      if (tfsf_in && on_face (p.face[2], z))
        zface |= 1u << j;
#pragma unroll
      for (int k = 0; k < 6; ++k)
        if (z >= p.ilo[k][2] && z < p.ihi[k][2])
          zin |= 1u << (4 * k + j);
    }
#pragma unroll
    for (int k = 0; k < 6; ++k)
      if (y >= p.ilo[k][1] && y < p.ihi[k][1])
        yin |= 1u << k;
    const bool yface = tfsf_in && on_face (p.face[1], y);
    const int zr = z0 + TZ;   // z ring cell (lane 31)
    const bool ring_lane = lane == 31 && w < WY - 1;

    float hp[3][4];           // H_old(x - 1) on the lane's cells
    float ep[3][4] = {};      // E_new(x - 1) on the lane's cells
    float hpr = 0.f;          // lane 31: Hz_old(x - 1) on the z ring cell
    float rxp = 0.f, ryp = 0.f;   // lane 31: Ex_new, Ey_new(x - 1) on the z ring cell
    // yface / zface only matter when the corrections run inside the sweep
    // One plane: stage st (= plane index mod 3, as every item restarts the
    // pipeline at stage 0) and exchange buffer st; kFull includes the PML,
    // in-sweep TF/SF and point-source code, the lean form is straight-line.
    auto plane = [&] (int i, auto st_c, auto full_c) __attribute__ ((always_inline)) -> bool {
      const unsigned st = st_c;       // a compile-time constant on the lean path
      const unsigned nbuf = st;
      constexpr bool kFull = decltype (full_c)::value;
      const int x = xa - 1 + i;
        if (!mbar_wait (bar + 8 * st, (phase >> st) & 1u))
        {
          s_abort[i & 1] = 1;
          atomicOr (err, 4);
        }
        phase ^= 1u << st;
        const int amode = kFull ? aux_mode (x, y0, zpml, nar_ok) : (MODE == 1 ? 1 : (MODE == 3 ? 2 : 0));
        const int apitch = amode == 2 ? PW : AN;
        const int acol = amode == 2 ? zl : zl - az0;      // only read on lanes with PML cells
        const unsigned char *stg = smem + st * L::STAGE;
        const T *sH = reinterpret_cast<const T *> (stg);
        const T *sE = reinterpret_cast<const T *> (stg + L::OFF_E);
        const float *P0 = reinterpret_cast<const float *> (stg + L::OFF_P);
        const float *P1 = P0 + PS;
        const float *A = reinterpret_cast<const float *> (stg + L::OFF_A);
        float *N = reinterpret_cast<float *> (smem + L::OFF_N + nbuf * 2 * L::P_B);

        float hc[3][4];
#pragma unroll
        for (int c = 0; c < 3; ++c)
          Vec<T>::ld4 (sH + c * HS + (w + 1) * HW + HZ + zl, hc[c]);
        const float hzr = Vec<T>::ld1 (sH + 2 * HS + (w + 1) * HW + HZ + TZ);
        // PML masks and auxiliaries of H(x - 1) for the H step (the stage is
        // refilled after the barrier)
        const int xh = x - 1;
        unsigned pmh[3] = {0u, 0u, 0u};
        float ha[3][4];
        if (amode && i > 1 && own_row && zupd)
        {
#pragma unroll
          for (int c = 0; c < 3; ++c)
          {
            const int k = 3 + c;
            const bool xy = xh >= p.ilo[k][0] && xh < p.ihi[k][0] && ((yin >> k) & 1u);
            pmh[c] = zupd & ~((xy ? zin : 0u) >> (4 * k)) & 15u;
            if (pmh[c] && !(MODE == 1 && c == 0))
              lds4f (A + (3 + c) * PS + w * apitch + acol, ha[c]);
          }
        }
        float en[3][4];           // E_new(x)
        float rx = 0.f, ry = 0.f; // lane 31: E_new(x) on the z ring cell

        if (i > 0)
        {
          // ================= E_new(x) on every row of the CTA (ring row included)
          const bool rowupd = x <= nx - 2 && yupd;
          const unsigned upd = rowupd ? zupd : 0u;
          const size_t id = (size_t) x * sx + rowoff;
          // PML cells of Ex..Ez on this lane and their auxiliaries (issued
          // first so that global reads overlap the curl arithmetic)
          unsigned pm[3] = {0u, 0u, 0u};
          float xo[3][4];
          if (amode && upd)
          {
#pragma unroll
            for (int k = 0; k < 3; ++k)
            {
              const bool xy = x >= p.ilo[k][0] && x < p.ihi[k][0] && ((yin >> k) & 1u);
              pm[k] = upd & ~((xy ? zin : 0u) >> (4 * k)) & 15u;
              if (pm[k] && !(MODE == 1 && k == 0))
                lds4f (A + k * PS + w * apitch + acol, xo[k]);
            }
          }
          float hzm[4], hxym[4], eo[3][4];
          Vec<T>::ld4 (sH + 2 * HS + w * HW + HZ + zl, hzm);
          Vec<T>::ld4 (sH + 0 * HS + w * HW + HZ + zl, hxym);
          const float hym1 = Vec<T>::ld1 (sH + 1 * HS + (w + 1) * HW + HZ + zl - 1);
          const float hxm1 = Vec<T>::ld1 (sH + 0 * HS + (w + 1) * HW + HZ + zl - 1);
#pragma unroll
          for (int c = 0; c < 3; ++c)
            Vec<T>::ld4 (sE + c * ES + w * EW + zl, eo[c]);
          float ix[4], iy[4], iz[4];
          if (has_eps)
          {
            float e0[4], ex1[4], ey1[4];
            lds4f (P0 + w * PW + zl, e0);
            lds4f (P1 + w * PW + zl, ex1);
            lds4f (P0 + min (w + 1, WY - 1) * PW + zl, ey1);
            const float ez1 = P0[w * PW + zl + 4];
#pragma unroll
            for (int j = 0; j < 4; ++j)
            {
              ix[j] = __fdividef (2.f, e0[j] + ex1[j]);
              iy[j] = __fdividef (2.f, e0[j] + ey1[j]);
              iz[j] = __fdividef (2.f, e0[j] + (j < 3 ? e0[j + 1] : ez1));
            }
          }
          else
          {
#pragma unroll
            for (int j = 0; j < 4; ++j)
              ix[j] = iy[j] = iz[j] = 1.f;
          }
          float cx[4], cy[4], cz[4];
#pragma unroll
          for (int j = 0; j < 4; ++j)
          {
            const float hyl = j ? hc[1][j - 1] : hym1;
            const float hxl = j ? hc[0][j - 1] : hxm1;
            cx[j] = (hc[2][j] - hzm[j]) - (hc[1][j] - hyl);
            cy[j] = (hc[0][j] - hxl) - (hc[2][j] - hp[2][j]);
            cz[j] = (hc[1][j] - hp[1][j]) - (hc[0][j] - hxym[j]);
          }
          const bool xface = kFull && tfsf_in && on_face (p.face[0], x);
          const unsigned fm = (xface || yface) ? upd : (zface & upd);
          if (fm)
          {
#pragma unroll
            for (int j = 0; j < 4; ++j)
              if ((fm >> j) & 1u)
              {
                cx[j] += tfsf_curl_cold (&p, 0, p.inc_h, err, x, y, zc + j);
                cy[j] += tfsf_curl_cold (&p, 1, p.inc_h, err, x, y, zc + j);
                cz[j] += tfsf_curl_cold (&p, 2, p.inc_h, err, x, y, zc + j);
              }
          }
          const bool store_e = own_row && x <= xb && lane_ok;
          if constexpr (MODE == 1)
          {
            float xn[4];
            zedge_vec<0> (tabs.z, zl, S, upd, pm[0], xo[0], cx, ix, eo[0], en[0], xn);
            zedge_vec<1> (tabs.z, zl, S, upd, pm[1], xo[1], cy, iy, eo[1], en[1], xn);
            if (pm[1] && store_e)
              Vec<float>::st4 (p.aux_new[1] + id, xn);
            zedge_vec<2> (tabs.z, zl, S, upd, pm[2], xo[2], cz, iz, eo[2], en[2], xn);
            if (pm[2] && store_e)
              Vec<float>::st4 (p.aux_new[2] + id, xn);
          }
          else
          {
#pragma unroll
            for (int j = 0; j < 4; ++j)
            {
              const bool u = (upd >> j) & 1u;
              en[0][j] = u ? eo[0][j] + (S * ix[j]) * cx[j] : eo[0][j];
              en[1][j] = u ? eo[1][j] + (S * iy[j]) * cy[j] : eo[1][j];
              en[2][j] = u ? eo[2][j] + (S * iz[j]) * cz[j] : eo[2][j];
            }
            if (pm[0])
            {
              float xn[4];
              pml_vec<0, WY> (tabs, S, w, i, zl, pm[0], xo[0], cx, ix, eo[0], en[0], xn);
              if (store_e)
                Vec<float>::st4 (p.aux_new[0] + id, xn);
            }
            if (pm[1])
            {
              float xn[4];
              pml_vec<1, WY> (tabs, S, w, i, zl, pm[1], xo[1], cy, iy, eo[1], en[1], xn);
              if (store_e)
                Vec<float>::st4 (p.aux_new[1] + id, xn);
            }
            if (pm[2])
            {
              float xn[4];
              pml_vec<2, WY> (tabs, S, w, i, zl, pm[2], xo[2], cz, iz, eo[2], en[2], xn);
              if (store_e)
                Vec<float>::st4 (p.aux_new[2] + id, xn);
            }
          }
          if (kFull && (p.ps_mask & 7) && rowupd && x == p.ps[0] && y == p.ps[1] && p.ps[2] >= zc && p.ps[2] < zc + 4)
          {
            const float v = (float) p.src[p.src_index];
            const int j = p.ps[2] - zc;
#pragma unroll
            for (int c = 0; c < 3; ++c)
              if (p.ps_mask & (1 << c))
              {
#pragma unroll
                for (int jj = 0; jj < 4; ++jj)
                  if (jj == j)
                    en[c][jj] = v;
              }
          }
          if (store_e)
          {
#pragma unroll
            for (int c = 0; c < 3; ++c)
              Vec<T>::st4 (reinterpret_cast<T *> (p.e_new[c]) + id, en[c]);
          }
          // Ex and Ez rows for the H step of the warp below (its y + 1 neighbours)
          sts4f (N + 0 * PS + w * PW + zl, en[0]);
          sts4f (N + 1 * PS + w * PW + zl, en[2]);

          // z ring: Ex and Ey at z0 + 128 for H of lane 31's last cell
          if (ring_lane && zr <= nz - 1)
          {
            rx = Vec<T>::ld1 (sE + 0 * ES + w * EW + TZ);
            ry = Vec<T>::ld1 (sE + 1 * ES + w * EW + TZ);
            if (rowupd && zr <= nz - 2)
            {
              const float hz = hzr;
              const float hzym = Vec<T>::ld1 (sH + 2 * HS + w * HW + HZ + TZ);
              const float hy = Vec<T>::ld1 (sH + 1 * HS + (w + 1) * HW + HZ + TZ);
              const float hx = Vec<T>::ld1 (sH + 0 * HS + (w + 1) * HW + HZ + TZ);
              float crx = (hz - hzym) - (hy - hc[1][3]);
              float cry = (hx - hc[0][3]) - (hz - hpr);
              float irx = 1.f, iry = 1.f;
              if (has_eps)
              {
                const float e0 = P0[w * PW + TZ];
                irx = __fdividef (2.f, e0 + P1[w * PW + TZ]);
                iry = __fdividef (2.f, e0 + P0[(w + 1) * PW + TZ]);
              }
              if (kFull && tfsf_in && (xface || yface || on_face (p.face[2], zr)))
              {
                crx += tfsf_curl_cold (&p, 0, p.inc_h, err, x, y, zr);
                cry += tfsf_curl_cold (&p, 1, p.inc_h, err, x, y, zr);
              }
              const bool in0 = x >= p.ilo[0][0] && x < p.ihi[0][0] && (yin & 1u) && zr >= p.ilo[0][2] &&
                               zr < p.ihi[0][2];
              const bool in1 = x >= p.ilo[1][0] && x < p.ihi[1][0] && (yin & 2u) && zr >= p.ilo[1][2] &&
                               zr < p.ihi[1][2];
              const int rcol = amode == 2 ? TZ : TZ - az0;
              if constexpr (MODE == 1)
              {
                const float *tz = tabs.z;
                const float xo1 = in1 ? 0.f : A[1 * PS + w * apitch + rcol];
                rx = fmaf (irx * tz[1 * PW + TZ], crx, tz[0 * PW + TZ] * rx);
                ry = fmaf (tz[3 * PW + TZ] * iry, cry, fmaf (tz[2 * PW + TZ] * iry, xo1, ry));
              }
              else
              {
                if (amode && !in0)
                  rx = pml_one<0, WY> (tabs, S, w, i, TZ, A[0 * PS + w * apitch + rcol], crx, irx, rx);
                else
                  rx = rx + (S * irx) * crx;
                if (amode && !in1)
                  ry = pml_one<1, WY> (tabs, S, w, i, TZ, A[1 * PS + w * apitch + rcol], cry, iry, ry);
                else
                  ry = ry + (S * iry) * cry;
              }
              if (kFull && (p.ps_mask & 3) && x == p.ps[0] && y == p.ps[1] && zr == p.ps[2])
              {
                const float v = (float) p.src[p.src_index];
                if (p.ps_mask & 1)
                  rx = v;
                if (p.ps_mask & 2)
                  ry = v;
              }
            }
          }
        }

        __syncthreads ();
        if (s_abort[i & 1])
        {
          // wait (bounded) for the copies still in flight into the other stages
          aborted = true;
          if (leader)
            for (int k = 1; k < NST && i + k < np; ++k)
            {
              const unsigned so = (st + k) % NST;
              mbar_wait (bar + 8 * so, (phase >> so) & 1u);
            }
          return false;
        }
        if (leader && i + NST < np)
          issue (st, x + NST, z0, y0,
                 MODE == 0 ? 0 : (MODE == 1 ? 1 : (MODE == 3 ? 2 : aux_mode (x + NST, y0, zpml, nar_ok))), az0);

        if (i > 1 && own_row)
        {
          // ================= H_new(x - 1) on the owned rows
          const size_t idh = (size_t) xh * sx + rowoff;
          const float *Np =
              reinterpret_cast<const float *> (smem + L::OFF_N + (nbuf == 0 ? 2u : nbuf - 1u) * 2 * L::P_B);
          float exy[4], ezy[4];
          lds4f (Np + 0 * PS + (w + 1) * PW + zl, exy);
          lds4f (Np + 1 * PS + (w + 1) * PW + zl, ezy);
          float exz = __shfl_down_sync (kLanes, ep[0][0], 1);
          float eyz = __shfl_down_sync (kLanes, ep[1][0], 1);
          if (lane == 31)
          {
            exz = rxp;
            eyz = ryp;
          }
          float ax[4], ay[4], az[4], hn[3][4];
#pragma unroll
          for (int j = 0; j < 4; ++j)
          {
            const float eyn = j < 3 ? ep[1][j + 1] : eyz;
            const float exn = j < 3 ? ep[0][j + 1] : exz;
            ax[j] = (eyn - ep[1][j]) - (ezy[j] - ep[2][j]);
            ay[j] = (en[2][j] - ep[2][j]) - (exn - ep[0][j]);
            az[j] = (exy[j] - ep[0][j]) - (en[1][j] - ep[1][j]);
          }
          const bool xface = kFull && tfsf_in && on_face (p.face[0], xh);
          const unsigned fm = (xface || yface) ? zupd : (zface & zupd);
          if (fm)
          {
#pragma unroll
            for (int j = 0; j < 4; ++j)
              if ((fm >> j) & 1u)
              {
                ax[j] += tfsf_curl_cold (&p, 3, p.inc_e, err, xh, y, zc + j);
                ay[j] += tfsf_curl_cold (&p, 4, p.inc_e, err, xh, y, zc + j);
                az[j] += tfsf_curl_cold (&p, 5, p.inc_e, err, xh, y, zc + j);
              }
          }
          if constexpr (MODE == 1)
          {
            float xn[4];
            zedge_vec<3> (tabs.z, zl, S, zupd, pmh[0], ha[0], ax, one4, hp[0], hn[0], xn);
            zedge_vec<4> (tabs.z, zl, S, zupd, pmh[1], ha[1], ay, one4, hp[1], hn[1], xn);
            if (pmh[1] && lane_ok)
              Vec<float>::st4 (p.aux_new[4] + idh, xn);
            zedge_vec<5> (tabs.z, zl, S, zupd, pmh[2], ha[2], az, one4, hp[2], hn[2], xn);
            if (pmh[2] && lane_ok)
              Vec<float>::st4 (p.aux_new[5] + idh, xn);
          }
          else
          {
#pragma unroll
            for (int j = 0; j < 4; ++j)
            {
              const bool u = (zupd >> j) & 1u;
              hn[0][j] = u ? hp[0][j] + S * ax[j] : hp[0][j];
              hn[1][j] = u ? hp[1][j] + S * ay[j] : hp[1][j];
              hn[2][j] = u ? hp[2][j] + S * az[j] : hp[2][j];
            }
            if (pmh[0])
            {
              float xn[4];
              pml_vec<3, WY> (tabs, S, w, i - 1, zl, pmh[0], ha[0], ax, one4, hp[0], hn[0], xn);
              if (lane_ok)
                Vec<float>::st4 (p.aux_new[3] + idh, xn);
            }
            if (pmh[1])
            {
              float xn[4];
              pml_vec<4, WY> (tabs, S, w, i - 1, zl, pmh[1], ha[1], ay, one4, hp[1], hn[1], xn);
              if (lane_ok)
                Vec<float>::st4 (p.aux_new[4] + idh, xn);
            }
            if (pmh[2])
            {
              float xn[4];
              pml_vec<5, WY> (tabs, S, w, i - 1, zl, pmh[2], ha[2], az, one4, hp[2], hn[2], xn);
              if (lane_ok)
                Vec<float>::st4 (p.aux_new[5] + idh, xn);
            }
          }
          if (kFull && (p.ps_mask & 56) && xh == p.ps[0] && y == p.ps[1] && p.ps[2] >= zc && p.ps[2] < zc + 4)
          {
            const float v = (float) p.src[p.src_index + 1] * p.ps_scale_h;
            const int j = p.ps[2] - zc;
#pragma unroll
            for (int c = 0; c < 3; ++c)
              if (p.ps_mask & (8 << c))
              {
#pragma unroll
                for (int jj = 0; jj < 4; ++jj)
                  if (jj == j)
                    hn[c][jj] = v;
              }
          }
          if (lane_ok)
          {
#pragma unroll
            for (int c = 0; c < 3; ++c)
              Vec<T>::st4 (reinterpret_cast<T *> (p.h_new[c]) + idh, hn[c]);
          }
        }

#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
          for (int j = 0; j < 4; ++j)
          {
            hp[c][j] = hc[c][j];
            ep[c][j] = en[c][j];
          }
        hpr = hzr;
        rxp = rx;
        ryp = ry;
        return true;
    };
    if (MODE != 2)
    {
      // stage and exchange buffer as compile-time constants
      using S0 = std::integral_constant<unsigned, 0>;
      using S1 = std::integral_constant<unsigned, 1>;
      using S2 = std::integral_constant<unsigned, 2>;
      for (int i = 0; i < np; i += 3)
      {
        if (!plane (i, S0{}, std::false_type{}))
          break;
        if (i + 1 < np && !plane (i + 1, S1{}, std::false_type{}))
          break;
        if (i + 2 < np && !plane (i + 2, S2{}, std::false_type{}))
          break;
      }
    }
    else
    {
      for (int i = 0; i < np; ++i)
        if (!plane (i, (unsigned) (i % 3), std::true_type{}))
          break;
    }
    if (aborted)
      break;
  }

  if (leader)
  {
    __threadfence ();
    const unsigned long long done = atomicAdd (wk.ctr + 2 * MODE + 1, 1ull);
    if (done == gridDim.x - 1)
    {
      atomicExch (wk.ctr + 2 * MODE, 0ull);
      atomicExch (wk.ctr + 2 * MODE + 1, 0ull);
    }
  }
}

// ------------------------------------------------------ TF/SF post pass

// Sum of the TF/SF terms of component k in mask m at (x, y, z): the terms
// of tfsf_curl that cover the cell, in the same order, without the box tests.
__device__ __forceinline__ float tfsf_terms (const FusedParams &p, int k, unsigned m, const double *inc, int *err,
                                             int x, int y, int z)
{
  const CompDev &c = p.comp[k];
  float d = 0.f;
#pragma unroll
  for (int t = 0; t < kMaxTerms; ++t)
    if ((m >> t) & 1u)
    {
      const TermDev &tm = c.term[t];
      const double diff =
          inc_at (p.g, inc, p.inc_len, err, tm.inc_comp, x + tm.aux[0], y + tm.aux[1], z + tm.aux[2]);
      const float dv = (float) (diff * tm.negate) * p.inc_scale[tm.inc_comp];
      d += (tm.slot == 0 || tm.slot == 3) ? dv : -dv;
    }
  return d;
}

// Cell of band box b taken by this thread (false past the box's end).
__device__ __forceinline__ bool band_cell (const BandBox &b, int first, int &x, int &y, int &z)
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

// The sweep ran without TF/SF, so on the band around the faces its E_new
// lacks (S im) dE for every corrected E cell and its H_new lacks
// S (curl of that dE + the H-side correction).  Both are linear in the
// correction, so adding them afterwards gives the corrected step (PML-free
// cells only, which the host guarantees).  One thread per band cell touches
// only its own cell; the E corrections of the +x / +y / +z neighbours are
// recomputed from the box's neighbour masks, never read, so there are no
// races.
template <typename T>
__global__ void __launch_bounds__ (256) tfsf_post_kernel (const __grid_constant__ FusedParams p, const BandBox *boxes,
                                                          const int2 *blk, int *err)
{
  const int2 bk = blk[blockIdx.x];
  const BandBox b = boxes[bk.x];
  int x, y, z;
  if (!band_cell (b, bk.y, x, y, z))
    return;
  const int nx = p.g.n[0], ny = p.g.n[1], nz = p.g.n[2];
  const size_t sx = (size_t) ny * nz;
  const float S = p.courant;
  // correction of E component k at (cx, cy, cz) from its terms in mask m:
  // zero where the step does not update the cell and on the point source
  // (band cells and their neighbours are >= 1 on every axis)
  auto de = [&] (int k, unsigned m, int cx, int cy, int cz) -> float {
    if (!m || cx > nx - 2 || cy > ny - 2 || cz > nz - 2)
      return 0.f;
    if (((p.ps_mask >> k) & 1) && cx == p.ps[0] && cy == p.ps[1] && cz == p.ps[2])
      return 0.f;
    const float d = tfsf_terms (p, k, m, p.inc_h, err, cx, cy, cz);
    if (d == 0.f)
      return 0.f;
    float im = 1.f;
    if (p.eps)
    {
      const size_t c = (size_t) cx * sx + (size_t) cy * nz + cz;
      const size_t st = k == 0 ? sx : (k == 1 ? (size_t) nz : 1);
      im = __fdividef (2.f, p.eps[c] + p.eps[c + st]);
    }
    return (S * im) * d;
  };
  auto em = [] (unsigned mask, int k) { return (mask >> (4 * k)) & 15u; };
  const size_t id = (size_t) x * sx + (size_t) y * nz + z;
  const float d0 = de (0, em (b.mask, 0), x, y, z), d1 = de (1, em (b.mask, 1), x, y, z),
              d2 = de (2, em (b.mask, 2), x, y, z);
  const float dd[3] = {d0, d1, d2};
#pragma unroll
  for (int k = 0; k < 3; ++k)
    if (dd[k] != 0.f)
    {
      T *f = reinterpret_cast<T *> (p.e_new[k]) + id;
      *f = (T) ((float) *f + dd[k]);
    }
  const unsigned hm[3] = {em (b.mask, 3), em (b.mask, 4), em (b.mask, 5)};
  const float a[3] = {
      (de (1, em (b.nmask[2], 1), x, y, z + 1) - d1) - (de (2, em (b.nmask[1], 2), x, y + 1, z) - d2) +
          (hm[0] ? tfsf_terms (p, 3, hm[0], p.inc_e, err, x, y, z) : 0.f),
      (de (2, em (b.nmask[0], 2), x + 1, y, z) - d2) - (de (0, em (b.nmask[2], 0), x, y, z + 1) - d0) +
          (hm[1] ? tfsf_terms (p, 4, hm[1], p.inc_e, err, x, y, z) : 0.f),
      (de (0, em (b.nmask[1], 0), x, y + 1, z) - d0) - (de (1, em (b.nmask[0], 1), x + 1, y, z) - d1) +
          (hm[2] ? tfsf_terms (p, 5, hm[2], p.inc_e, err, x, y, z) : 0.f)};
  const bool at_src = x == p.ps[0] && y == p.ps[1] && z == p.ps[2];
#pragma unroll
  for (int m = 0; m < 3; ++m)
    if (a[m] != 0.f && !(at_src && ((p.ps_mask >> (3 + m)) & 1)))
    {
      T *f = reinterpret_cast<T *> (p.h_new[m]) + id;
      *f = (T) ((float) *f + S * a[m]);
    }
}

}  // namespace

// ------------------------------------------------------------------ host side

namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode_fn ()
{
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once (once, [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint ("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000> (f);
  });
  return fn;
}

}  // namespace

// 3-D map over an (nx, ny, nz) array, z fastest, box bw x bh x 1
bool make_map (CUtensorMap &m, const void *base, bool half, const int n[3], int bw, int bh)
{
  // L2 fetch granularity of the copies: 64 bytes measured best at 512^3
  // with the concurrent class launches (1.673 ms per step against 1.681 for
  // 128 bytes and none, 1.700 for 256)
  constexpr CUtensorMapL2promotion promo = CU_TENSOR_MAP_L2_PROMOTION_L2_64B;
  auto fn = encode_fn ();
  if (!fn)
    return false;
  const cuuint64_t es = half ? 2 : 4;
  cuuint64_t dims[3] = {(cuuint64_t) n[2], (cuuint64_t) n[1], (cuuint64_t) n[0]};
  cuuint64_t strides[2] = {(cuuint64_t) n[2] * es, (cuuint64_t) n[2] * (cuuint64_t) n[1] * es};
  cuuint32_t box[3] = {(cuuint32_t) bw, (cuuint32_t) bh, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn (&m, half ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
                   const_cast<void *> (base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_NONE, promo, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

namespace {

template <typename T, int WY>
std::string plan_t (SweepPlan &pl, const FusedParams &p, void *const e[2][3], void *const h[2][3],
                    float *const aux[2][6], const float *eps, int sm_count)
{
  using L = Smem<T, WY>;
  const bool half = sizeof (T) == 2;
  for (int b = 0; b < 2; ++b)
  {
    SweepMaps &m = pl.maps[b];
    for (int c = 0; c < 3; ++c)
      if (!make_map (m.h[c], h[b][c], half, p.g.n, L::HW, WY + 1) ||
          !make_map (m.e[c], e[b][c], half, p.g.n, L::EW, WY))
        return "tensor map encoding failed";
    // descriptors the kernel never uses are copies of a valid one
    if (eps)
    {
      if (!make_map (m.eps, eps, false, p.g.n, PW, WY))
        return "tensor map encoding failed";
    }
    else
      m.eps = m.e[0];
    for (int k = 0; k < 6; ++k)
    {
      if (p.use_pml)
      {
        if (!aux[b][k] || !make_map (m.aux[k], aux[b][k], false, p.g.n, PW, WY) ||
            !make_map (m.auxn[k], aux[b][k], false, p.g.n, L::AN, WY))
          return "tensor map encoding failed";
      }
      else
        m.aux[k] = m.auxn[k] = m.e[0];
    }
  }
  int per_sm = 0;
  for (int mode = 0; mode < 4; ++mode)
  {
    auto kern = mode == 0   ? sweep3d_kernel<T, WY, 0>
                : mode == 1 ? sweep3d_kernel<T, WY, 1>
                : mode == 2 ? sweep3d_kernel<T, WY, 2>
                            : sweep3d_kernel<T, WY, 3>;
    if (cudaFuncSetAttribute (kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) L::TOTAL) != cudaSuccess)
    {
      cudaGetLastError ();
      return "shared memory request refused";
    }
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor (&n, kern, 32 * WY, L::TOTAL) != cudaSuccess || n < 1)
    {
      cudaGetLastError ();
      return "kernel does not fit on an SM";
    }
    per_sm = mode ? std::min (per_sm, n) : n;
  }
  pl.smem = L::TOTAL;
  pl.ctas = sm_count * per_sm;
  return "";
}

template <typename T, int WY>
int launch_t (const SweepPlan &pl, int set, const FusedParams &p, int *err, cudaStream_t s, const SweepStreams &ss)
{
  // on side streams the next class's CTAs take the SMs as the previous
  // class's persistent CTAs run out of items
  constexpr unsigned sm = Smem<T, WY>::TOTAL;
  const bool conc = ss.side[0] && ss.side[1];
  cudaStream_t s1 = s, s0 = s;
  if (conc)
  {
    cudaEventRecord (ss.fork, s);
    cudaStreamWaitEvent (ss.side[0], ss.fork, 0);
    cudaStreamWaitEvent (ss.side[1], ss.fork, 0);
    s1 = ss.side[0];
    s0 = ss.side[1];
  }
  int n = 0;
  if (pl.items[2] > 0)
  {
    sweep3d_kernel<T, WY, 2><<<pl.ctas, dim3 (32, WY), sm, s>>> (pl.maps[set], p, pl.work, err);
    ++n;
  }
  // launch order of the PML (3), z-edge (1) and lean (0) classes on s, s1,
  // s0: z-edge, lean, PML measured best at 512^3 (1.680 ms per step against
  // 1.689 for PML, z-edge, lean and 1.723 for PML, lean, z-edge)
  constexpr char order[4] = "103";
  const cudaStream_t on[3] = {s, s1, s0};
  for (int j = 0; j < 3; ++j)
  {
    const int c = order[j] - '0';
    if (pl.items[c] <= 0)
      continue;
    if (c == 3)
      sweep3d_kernel<T, WY, 3><<<pl.ctas, dim3 (32, WY), sm, on[j]>>> (pl.maps[set], p, pl.work, err);
    else if (c == 1)
      sweep3d_kernel<T, WY, 1><<<pl.ctas, dim3 (32, WY), sm, on[j]>>> (pl.maps[set], p, pl.work, err);
    else
      sweep3d_kernel<T, WY, 0><<<pl.ctas, dim3 (32, WY), sm, on[j]>>> (pl.maps[set], p, pl.work, err);
    ++n;
  }
  if (conc)
  {
    cudaEventRecord (ss.join[0], ss.side[0]);
    cudaEventRecord (ss.join[1], ss.side[1]);
    cudaStreamWaitEvent (s, ss.join[0], 0);
    cudaStreamWaitEvent (s, ss.join[1], 0);
  }
  return n;
}

}  // namespace

void sweep3d_items (const FusedParams &p, int wy, int chunk, SweepWork &w)
{
  const int *n = p.g.n;
  w.nzt = (n[2] - 1 + TZ - 1) / TZ;
  w.nyt = (n[1] - 2 + wy - 2) / (wy - 1);
  if (p.use_pml && chunk > MAXC)
    chunk = MAXC;   // the item's x coefficient table holds MAXC + 2 planes
  chunk = std::max (chunk, (n[0] - 2 + kMaxChunks - 1) / kMaxChunks);
  w.chunk = chunk;
  // x segments: the planes where every component is PML-free (E on
  // x .. x + 1, H on x) form the middle segment, so that no item mixes PML
  // and interior planes; each segment is split into near-equal chunks
  int lo = 1, hi = n[0] - 2;   // interior segment [lo, hi]
  if (p.use_pml)
  {
    for (int k = 0; k < 6; ++k)
    {
      lo = std::max (lo, p.ilo[k][0]);
      hi = std::min (hi, k < 3 ? p.ihi[k][0] - 2 : p.ihi[k][0] - 1);
    }
  }
  std::vector<int> seg = {1};
  if (lo > 1 && lo <= hi)
    seg.push_back (lo);
  if (hi + 1 <= n[0] - 2 && lo <= hi)
    seg.push_back (hi + 1);
  seg.push_back (n[0] - 1);
  w.nch = 0;
  w.xcut[0] = 1;
  for (size_t sg = 0; sg + 1 < seg.size (); ++sg)
  {
    const int len = seg[sg + 1] - seg[sg];
    const int m = (len + chunk - 1) / chunk;
    for (int j = 1; j <= m; ++j)
      w.xcut[++w.nch] = seg[sg] + (int) ((long long) len * j / m);
  }
  w.nitems = w.nzt * w.nyt * w.nch;
  w.list = nullptr;
  w.nlist = 0;
}

std::string sweep3d_plan (SweepPlan &plan, const FusedParams &p, void *const e[2][3], void *const h[2][3],
                          float *const aux[2][6], const float *eps, int sm_count, int wy, int chunk,
                          unsigned long long *ctr, bool lean)
{
  const int *n = p.g.n;
  if (p.g.drop != 0)
    return "2-D grid";
  const int unit = p.fp16 ? 8 : 4;
  if (n[2] % unit != 0)
    return "nz is not a multiple of one 16-byte unit";
  if (n[0] < 3 || n[1] < 3 || n[2] < 3)
    return "grid too small";
  if (wy != 8)
    return "unsupported CTA height";
  if (chunk < 1)
    return "bad x chunk";
  plan.wy = wy;
  std::string why = p.fp16 ? plan_t<__half, 8> (plan, p, e, h, aux, eps, sm_count)
                           : plan_t<float, 8> (plan, p, e, h, aux, eps, sm_count);
  if (!why.empty ())
    return why;
  sweep3d_items (p, wy, chunk, plan.work);
  if (p.use_pml && plan.work.chunk > MAXC)
    return "grid too long in x for the staged PML coefficients";
  plan.work.ctr = ctr;
  plan.work.lean = lean ? 1 : 0;
  const bool tfsf_in = p.use_tfsf && !p.tfsf_post;
  plan.items[0] = plan.items[1] = plan.items[2] = plan.items[3] = 0;
  for (int it = 0; it < plan.work.nitems; ++it)
    ++plan.items[sweep_item_class (p, plan.work, wy, it, tfsf_in)];
  if (plan.ctas > plan.work.nitems)
    plan.ctas = plan.work.nitems;
  return "";
}

std::string sweep3d_plan_list (SweepPlan &plan, const FusedParams &p, void *const e[2][3], void *const h[2][3],
                               float *const aux[2][6], const float *eps, int sm_count, const std::vector<int> &cuts,
                               const std::vector<int> &host_list, int *dev_list, unsigned long long *ctr,
                               cudaStream_t s)
{
  std::string why = sweep3d_plan (plan, p, e, h, aux, eps, sm_count, 8, 32, ctr, true);
  if (!why.empty ())
    return why;
  if (cuts.size () < 2 || cuts.size () > (size_t) kMaxChunks + 1 || cuts.front () != 1 ||
      cuts.back () != p.g.n[0] - 1)
    return "bad x cuts";
  SweepWork &w = plan.work;
  w.nch = (int) cuts.size () - 1;
  for (int j = 0; j <= w.nch; ++j)
    w.xcut[j] = cuts[j];
  for (int j = 0; j < w.nch; ++j)
    if (w.xcut[j + 1] <= w.xcut[j] || (p.use_pml && w.xcut[j + 1] - w.xcut[j] > MAXC))
      return "bad x cuts";
  w.chunk = 0;
  w.nitems = w.nzt * w.nyt * w.nch;
  for (int it : host_list)
    if (it < 0 || it >= w.nitems)
      return "item out of range";
  w.list = dev_list;
  w.nlist = (int) host_list.size ();
  if (!host_list.empty () &&
      cudaMemcpyAsync (dev_list, host_list.data (), host_list.size () * sizeof (int), cudaMemcpyHostToDevice, s) !=
          cudaSuccess)
    return "item list upload failed";
  const bool tfsf_in = p.use_tfsf && !p.tfsf_post;
  plan.items[0] = plan.items[1] = plan.items[2] = plan.items[3] = 0;
  for (int it : host_list)
    ++plan.items[sweep_item_class (p, w, 8, it, tfsf_in)];
  plan.ctas = std::min (plan.ctas, std::max (1, w.nlist));
  return "";
}

int launch_sweep3d (const SweepPlan &plan, int set, const FusedParams &p, int *err, cudaStream_t s,
                    const SweepStreams &ss)
{
  return p.fp16 ? launch_t<__half, 8> (plan, set, p, err, s, ss) : launch_t<float, 8> (plan, set, p, err, s, ss);
}

}  // namespace fdtdb

// --------------------------------------------------- TF/SF post pass (host)

namespace fdtdb {

std::string tfsf_band_boxes (const FusedParams &p, std::vector<BandBox> &boxes, std::vector<int2> &blk)
{
  struct Box
  {
    int lo[3], hi[3];
  };
  std::vector<Box> cand;
  const int *n = p.g.n;
  auto add = [&] (const TermDev &t, int shift_axis) {
    Box b;
    for (int a = 0; a < 3; ++a)
    {
      const int d = a == shift_axis ? 1 : 0;
      b.lo[a] = std::max (t.lo[a] - d, 1);
      b.hi[a] = std::min (t.hi[a] - d, n[a] - 1);
    }
    if (b.lo[0] < b.hi[0] && b.lo[1] < b.hi[1] && b.lo[2] < b.hi[2])
      cand.push_back (b);
  };
  for (int k = 0; k < 6; ++k)
    for (int t = 0; t < p.comp[k].nterms; ++t)
    {
      add (p.comp[k].term[t], -1);
      if (k < 3)
        for (int a = 0; a < 3; ++a)
          add (p.comp[k].term[t], a);
    }
  boxes.clear ();
  blk.clear ();
  if (cand.empty ())
    return "";
  // disjoint cover: compress coordinates (every term box edge is a cut, so
  // an elementary box lies wholly inside or outside each term), keep the
  // covered elementary boxes, merge runs along z with equal term masks
  std::vector<int> cut[3];
  for (const Box &b : cand)
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
  const size_t mx = cut[0].size () - 1, my = cut[1].size () - 1, mz = cut[2].size () - 1;
  // the elementary box (i, j, l), moved by +1 along axis sh (-1: not moved),
  // inside the box lo .. hi - 1
  auto inside = [&] (const int lo[3], const int hi[3], size_t i, size_t j, size_t l, int sh = -1) {
    const size_t ix[3] = {i, j, l};
    for (int a = 0; a < 3; ++a)
    {
      const int d = a == sh ? 1 : 0;
      if (cut[a][ix[a]] + d < lo[a] || cut[a][ix[a] + 1] + d > hi[a])
        return false;
    }
    return true;
  };
  auto covered = [&] (size_t i, size_t j, size_t l) {
    for (const Box &b : cand)
      if (inside (b.lo, b.hi, i, j, l))
        return true;
    return false;
  };
  // term masks of the elementary box (every component) or of the box moved
  // by +1 along sh (E components only); uniform over the box because the
  // term boxes and the E term boxes moved by -1 along each axis are all cut
  auto mask_of = [&] (size_t i, size_t j, size_t l, int sh = -1) {
    unsigned m = 0;
    for (int k = 0; k < (sh < 0 ? 6 : 3); ++k)
      for (int t = 0; t < p.comp[k].nterms; ++t)
        if (inside (p.comp[k].term[t].lo, p.comp[k].term[t].hi, i, j, l, sh))
          m |= 1u << (4 * k + t);
    return m;
  };
  auto masks_of = [&] (size_t i, size_t j, size_t l, unsigned m[4]) {
    m[0] = mask_of (i, j, l);
    for (int a = 0; a < 3; ++a)
      m[1 + a] = mask_of (i, j, l, a);
  };
  auto same = [] (const unsigned u[4], const unsigned v[4]) {
    return u[0] == v[0] && u[1] == v[1] && u[2] == v[2] && u[3] == v[3];
  };
  for (size_t i = 0; i < mx; ++i)
    for (size_t j = 0; j < my; ++j)
    {
      size_t l = 0;
      while (l < mz)
      {
        if (!covered (i, j, l))
        {
          ++l;
          continue;
        }
        unsigned m[4], me[4];
        masks_of (i, j, l, m);
        size_t e = l + 1;
        while (e < mz && covered (i, j, e) && (masks_of (i, j, e, me), same (m, me)))
          ++e;
        BandBox bb;
        bb.lo[0] = cut[0][i];
        bb.lo[1] = cut[1][j];
        bb.lo[2] = cut[2][l];
        bb.hi[0] = cut[0][i + 1];
        bb.hi[1] = cut[1][j + 1];
        bb.hi[2] = cut[2][e];
        bb.mask = m[0];
        for (int a = 0; a < 3; ++a)
          bb.nmask[a] = m[1 + a];
        // a band cell must not be a PML cell of any component
        for (int k = 0; k < 6; ++k)
          for (int a = 0; a < 3; ++a)
            if (p.use_pml && (bb.lo[a] < p.ilo[k][a] || bb.hi[a] > p.ihi[k][a]))
              return "the TF/SF band reaches into the PML";
        boxes.push_back (bb);
        l = e;
      }
    }
  for (size_t q = 0; q < boxes.size (); ++q)
  {
    const BandBox &bb = boxes[q];
    const long long cells = (long long) (bb.hi[0] - bb.lo[0]) * (bb.hi[1] - bb.lo[1]) * (bb.hi[2] - bb.lo[2]);
    if (cells >= (1ll << 31))
      return "TF/SF band box too large";
    for (long long f = 0; f < cells; f += 256)
      blk.push_back (make_int2 ((int) q, (int) f));
  }
  return "";
}

int launch_tfsf_post (const TfsfBand &band, const FusedParams &p, int *err, cudaStream_t s)
{
  if (band.cells <= 0 || band.nblk <= 0)
    return 0;
  if (p.fp16)
    tfsf_post_kernel<__half><<<band.nblk, 256, 0, s>>> (p, band.boxes, band.blk, err);
  else
    tfsf_post_kernel<float><<<band.nblk, 256, 0, s>>> (p, band.boxes, band.blk, err);
  return 1;
}

}  // namespace fdtdb
