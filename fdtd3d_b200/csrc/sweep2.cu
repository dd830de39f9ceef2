// sweep2.cu - two leapfrog time steps per pass over HBM (temporal blocking)
// for the 3-D FP32 and FP16-storage forms.
//
// The single-step sweep (sweep3d.cu) reads every field once and writes it
// once per step.  Here a CTA advances its tile by two steps in one sweep
// along x, so the fields cross HBM once per two steps:
//
//  * A CTA holds 16 warps, warp w on row Y + w, lane l on the two z cells
//    zs + 2l, zs + 2l + 1.  The tile's own cells are rows Y + 1 .. Y + 13 and
//    z cells zs + 2 .. zs + 61; the rest is halo.  The first step is computed
//    on the whole 16 x 64 tile, and each later half-step loses one row or
//    column on the side its stencil reaches (H needs E at y + 1 / z + 1, E
//    needs H at y - 1 / z - 1), so the second step is exact on the own cells
//    and the halo costs recomputation, never communication.
//  * Per plane x, one elected thread streams H(x) (with the y - 1 row and a
//    16-byte z halo), E(x), eps(x) and eps(x + 1) of the old buffer set into
//    shared memory with cp.async.bulk.tensor, three stages deep (bounded
//    mbarrier waits).  Iteration x then computes E1(x), H1(x - 1) | barrier |
//    E2(x - 1), H2(x - 2), where E1, H1 are the first step's values and E2,
//    H2 the second's: one barrier per plane.  Neighbours along z come from
//    warp shuffles, along y from shared exchange rows (double-buffered by
//    plane parity) written one phase earlier, along x from registers carried
//    over from the previous plane.  Only E2 and H2 of the own cells go to
//    the new buffer set.
//  * CTAs are persistent and take (z tile, y tile, x chunk) items from an
//    atomic counter.
// The arithmetic of each half-step is the one-sweep kernel's (the same
// expressions in the same order), so two steps here equal two single steps.
#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <type_traits>
#include <vector>

#include "sweep2.h"
#include "tma.cuh"

namespace fdtdb {

namespace {

constexpr int NW = kTb2Warps;   // warps = rows per CTA
constexpr int ZW = kTb2Zw;      // z cells per warp row
constexpr int NST2 = 3;         // pipeline stages

template <typename T>
struct L2
{
  // z tiling: tile k's warp rows start at zs = ZOWN k - ZOFF (a multiple of
  // one 16-byte unit, as TMA requires) and own the cells
  // zs + 2 OLO .. zs + 2 OHI + 1 (lanes OLO .. OHI)
  static constexpr int ZOWN = sizeof (T) == 4 ? 60 : 56;
  static constexpr int ZOFF = sizeof (T) == 4 ? 4 : 8;
  static constexpr int OLO = sizeof (T) == 4 ? 1 : 2;
  static constexpr int OHI = OLO + ZOWN / 2 - 1;
  static constexpr int HZ = 16 / (int) sizeof (T);   // z halo: one 16-byte unit
  static constexpr int HW = ZW + HZ;                 // H row: zs - HZ .. zs + 63
  static constexpr int HR = NW + 1;                  // H rows: Y - 1 .. Y + 15
  static constexpr int EW = ZW;                      // E row: zs .. zs + 63
  static constexpr int ER = NW;                      // E rows: Y .. Y + 15
  static constexpr int PW = ZW + 4;                  // eps row (float): zs .. zs + 67
  static constexpr int PR = NW + 1;                  // eps rows: Y .. Y + 16
  static constexpr unsigned rnd (unsigned b) { return (b + 127u) / 128u * 128u; }
  static constexpr unsigned H_B = rnd (sizeof (T) * HW * HR);
  static constexpr unsigned E_B = rnd (sizeof (T) * EW * ER);
  static constexpr unsigned P_B = rnd (4u * PW * PR);
  static constexpr unsigned A_B = rnd (4u * ZW * NW);   // one auxiliary box (float): zs .. zs + 63 x Y .. Y + 15
  static constexpr unsigned OFF_E = 3 * H_B;
  static constexpr unsigned OFF_P = OFF_E + 3 * E_B;
  // z-edge class: old auxiliaries of Ey, Ez at x and Hy, Hz at x - 1
  static constexpr unsigned OFF_A = OFF_P + 2 * P_B;
  static constexpr unsigned STAGE = OFF_A + 4 * A_B;
  // exchange rows, NW x ZW floats each: XE1[parity][Ex, Ez],
  // XH1[parity][Hx, Hz], XE2[parity][Ex, Ez]
  static constexpr int XN = NW * ZW;
  static constexpr unsigned OFF_X = NST2 * STAGE;
  // z-edge class: the item's z coefficient pairs, pre-combined, per
  // component k and element e at [(2k + e) ZW + column]
  static constexpr unsigned OFF_T = OFF_X + 12u * 4u * XN;
  static constexpr unsigned OFF_BAR = OFF_T + rnd (4u * 12 * ZW);
  static constexpr unsigned TOTAL = OFF_BAR + 64 + 128;   // + room to align the base to 128 bytes
  // bytes each stage's copies deliver (full boxes, fill included)
  static constexpr unsigned TX_HE = 3u * sizeof (T) * HW * HR + 3u * sizeof (T) * EW * ER;
  static constexpr unsigned TX_P = 2u * 4u * PW * PR;
  static constexpr unsigned TX_A = 4u * 4u * ZW * NW;
};

template <typename T>
struct V2;

template <>
struct V2<float>
{
  static __device__ __forceinline__ void ld (const float *s, float v[2])
  {
    const float2 t = *reinterpret_cast<const float2 *> (s);
    v[0] = t.x;
    v[1] = t.y;
  }
  static __device__ __forceinline__ float ld1 (const float *s) { return *s; }
  static __device__ __forceinline__ void st (float *g, const float v[2])
  {
    __stcs (reinterpret_cast<float2 *> (g), make_float2 (v[0], v[1]));
  }
};

template <>
struct V2<__half>
{
  static __device__ __forceinline__ void ld (const __half *s, float v[2])
  {
    const float2 t = __half22float2 (*reinterpret_cast<const __half2 *> (s));
    v[0] = t.x;
    v[1] = t.y;
  }
  static __device__ __forceinline__ float ld1 (const __half *s) { return __half2float (*s); }
  static __device__ __forceinline__ void st (__half *g, const float v[2])
  {
    const __half2 h = __floats2half2_rn (v[0], v[1]);
    __stcs (reinterpret_cast<unsigned *> (g), *reinterpret_cast<const unsigned *> (&h));
  }
};

__device__ __forceinline__ void lds2 (const float *s, float v[2])
{
  V2<float>::ld (s, v);
}

__device__ __forceinline__ void sts2 (float *s, const float v[2])
{
  *reinterpret_cast<float2 *> (s) = make_float2 (v[0], v[1]);
}

// Auxiliary values of a lane's two cells (bits: which are PML cells; the
// pair starts on an 8-byte boundary).
__device__ __forceinline__ void store_aux (float *g, unsigned bits, const float v[2])
{
  if (bits == 3u)
    __stcs (reinterpret_cast<float2 *> (g), make_float2 (v[0], v[1]));
  else
  {
#pragma unroll
    for (int j = 0; j < 2; ++j)
      if ((bits >> j) & 1u)
        __stcs (g + j, v[j]);
  }
}

// ------------------------------------------------------------------ kernel

// Pair (0: ca1, sq1; 1: p5, q5; 2: g4p, g4m) of component k that runs along
// an axis.
__device__ __forceinline__ int pair_along (int k, int axis)
{
  return (k + 1) % 3 == axis ? 0 : ((k + 2) % 3 == axis ? 1 : 2);
}

// z-edge items (x and y interior for every component, PML cells only along
// z): the single-step kernel's branch-free form, in which only the z pair
// of each component differs from the sigma = 0 identity and the item's z
// table holds it pre-combined (zedge_pair in sweep3d.cu): for the pair
// (p5, q5) along z (Ex, Hx) F = p5 F + S q5 im curl (no auxiliary); for
// (ca1, sq1) (Ey, Hy) X_new = ca1 X + sq1 curl, F = F + ((ca1 - 1) X +
// sq1 curl) im; for (g4p, g4m) (Ez, Hz) X_new = X + S curl,
// F = F + ((g4p - g4m) X + S g4p curl) im, with X = 0 on cells that are not
// PML cells of the component.  With the identity values each form is the
// plain update F + (S im) curl bit for bit.  fn gets F_new on the updated
// cells (upd) and F elsewhere, xn X_new on the PML cells (pm), 0 elsewhere.
__device__ __forceinline__ void zedge_two (const float *Tz, int k, int zl, float S, unsigned upd, unsigned pm,
                                           const float xo[2], const float cu[2], const float im[2], const float fo[2],
                                           float fn[2], float xn[2])
{
  const int pz = pair_along (k, 2);
  float c0[2], c1[2];
  lds2 (Tz + (2 * k) * ZW + zl, c0);
  lds2 (Tz + (2 * k + 1) * ZW + zl, c1);
#pragma unroll
  for (int j = 0; j < 2; ++j)
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

// MODE 0 (lean): no cell of the item's extended region is a PML cell of any
// component.  MODE 2 (z edge): PML cells only along z; every lane runs the
// branch-free z-edge form (zedge_two), carries the first step's auxiliaries
// in registers to the second, and takes the old auxiliaries of the four
// components that keep one (Ey, Ez at x, Hy, Hz at x - 1) through the
// plane's TMA stage.  (Class 1, x or y PML cells, is left to the
// single-step kernels: the two-step plan refuses it.)
template <typename T, int MODE>
__global__ void __launch_bounds__ (32 * NW, 1)
    sweep2_kernel (const __grid_constant__ Sweep2Maps maps, const __grid_constant__ FusedParams p,
                   const Sweep2Work wk, int *err)
{
  using L = L2<T>;
  constexpr int HZ = L::HZ, HW = L::HW, EW = L::EW, PW = L::PW, XN = L::XN;
  constexpr int HS = L::H_B / sizeof (T), ES = L::E_B / sizeof (T), PS = L::P_B / sizeof (float);
  constexpr unsigned kLanes = 0xffffffffu;
  constexpr bool kZedge = MODE == 2;
  constexpr bool kAux = kZedge;   // PML masks and auxiliaries
  extern __shared__ __align__ (128) unsigned char smem_raw[];
  __shared__ int s_item;
  __shared__ int s_abort;

  const int lane = threadIdx.x, w = threadIdx.y;
  const bool leader = w == 0 && lane == 0;
  const int nx = p.g.n[0], ny = p.g.n[1], nz = p.g.n[2];
  const size_t sx = (size_t) ny * nz;
  const uint32_t raw = tma::smem_addr (smem_raw);
  const uint32_t sbase = (raw + 127u) & ~127u;
  unsigned char *const smem = smem_raw + (sbase - raw);
  const uint32_t bar = sbase + L::OFF_BAR;
  const bool has_eps = p.eps != nullptr;
  const float S = p.courant;
  float *const X = reinterpret_cast<float *> (smem + L::OFF_X);
  float *const Tab = reinterpret_cast<float *> (smem + L::OFF_T);

  if (leader)
  {
#pragma unroll
    for (int st = 0; st < NST2; ++st)
      tma::mbar_init (bar + 8 * st, 1);
    asm volatile ("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_abort = 0;
  }
  __syncthreads ();

  // stage st <- plane x of the tile at (zs, Y)
  auto issue = [&] (int st, int x, int zs, int Y) {
    const uint32_t s = sbase + st * L::STAGE;
    const uint32_t b = bar + 8 * st;
    tma::mbar_expect_tx (b, L::TX_HE + (has_eps ? L::TX_P : 0u) + (kAux ? L::TX_A : 0u));
    if (kAux)
    {
      // the components that keep an auxiliary in the z-edge form: Ey, Ez, Hy, Hz
#pragma unroll
      for (int q = 0; q < 4; ++q)
      {
        const int k = q < 2 ? 1 + q : 2 + q;
        tma::load_3d (s + L::OFF_A + q * L::A_B, &maps.aux[k], zs, Y, k < 3 ? x : x - 1, b);
      }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c)
      tma::load_3d (s + c * L::H_B, &maps.h[c], zs - HZ, Y - 1, x, b);
#pragma unroll
    for (int c = 0; c < 3; ++c)
      tma::load_3d (s + L::OFF_E + c * L::E_B, &maps.e[c], zs, Y, x, b);
    if (has_eps)
    {
      tma::load_3d (s + L::OFF_P, &maps.eps, zs, Y, x, b);
      tma::load_3d (s + L::OFF_P + L::P_B, &maps.eps, zs, Y, x + 1, b);
    }
  };

  unsigned phase = 0;   // bit s: parity of the next completion of stage s
  bool aborted = false;
  static_assert (MODE == 0 || MODE == 2, "item class");
  for (;;)
  {
    __syncthreads ();   // every thread has read the previous item's index
    if (leader)
      s_item = (int) atomicAdd (wk.ctr + 2 * MODE, 1ull);
    __syncthreads ();
    const int item = s_item;
    if (item >= wk.nitems)
      break;
    if (sweep2_item_class (p, wk, item) != MODE)
      continue;
    const int zt = item % wk.nzt;
    const int yt = (item / wk.nzt) % wk.nyt;
    const int ch = item / (wk.nzt * wk.nyt);
    const int zs = L::ZOWN * zt - L::ZOFF;   // first z cell of the warp rows
    const int Y = wk.yoff + kTb2Yown * yt;   // row of warp 0
    const int xa = wk.xcut[ch];
    const int xb = wk.xcut[ch + 1] - 1;
    const int np = xb - xa + 5;              // planes xa - 2 .. xb + 2

    if (leader)
    {
#pragma unroll
      for (int k = 0; k < NST2; ++k)
        issue (k, xa - 2 + k, zs, Y);
    }
    if constexpr (kZedge)
    {
      // the item's z pairs in the z-edge form (read after the first plane's
      // barrier)
      const int tid = w * 32 + lane;
      for (int q = tid; q < 6 * ZW; q += 32 * NW)
      {
        const int k = q / ZW, col = q % ZW, z = min (max (zs + col, 0), nz - 1), pz = pair_along (k, 2);
        const float a = __ldg (p.tab[k][2 * pz] + z), b = __ldg (p.tab[k][2 * pz + 1] + z);
        float c0, c1;
        if (pz == 1)
        {
          c0 = a;
          c1 = S * b;
        }
        else if (pz == 0)
        {
          c0 = a - 1.f;
          c1 = b;
        }
        else
        {
          c0 = S * a;
          c1 = a - b;
        }
        Tab[(2 * k) * ZW + col] = c0;
        Tab[(2 * k + 1) * ZW + col] = c1;
      }
    }
    // ---- per-lane constants of this item
    const int r = Y + w;
    const int zl = 2 * lane;
    const int zc = zs + zl;
    unsigned cupd = 0;   // bit j: cell zc + j of this row is updated (on an updated plane)
    if (r >= 1 && r <= ny - 2)
    {
#pragma unroll
      for (int j = 0; j < 2; ++j)
        if (zc + j >= 1 && zc + j <= nz - 2)
          cupd |= 1u << j;
    }
    const bool own = w >= 1 && w <= kTb2Yown && r < wk.yend && lane >= L::OLO && lane <= L::OHI && zc >= 0 && zc < nz;
    const size_t rowoff = (size_t) r * nz + zc;
    // y / z membership of this lane's cells in each component's sigma = 0
    // box: bit 2k + j (k = 0 .. 5, cell j) of yz_in
    unsigned yz_in = 0;
    if (kAux)
    {
#pragma unroll
      for (int k = 0; k < 6; ++k)
        if (r >= p.ilo[k][1] && r < p.ihi[k][1])
#pragma unroll
          for (int j = 0; j < 2; ++j)
            if (zc + j >= p.ilo[k][2] && zc + j < p.ihi[k][2])
              yz_in |= 1u << (2 * k + j);
    }
    // PML cells of the family (E: kb = 0, H: kb = 3) among this lane's
    // updated cells on plane xx: bit 2c + j for component kb + c, cell j
    auto pmask = [&] (int kb, int xx) -> unsigned {
      const unsigned u = (xx >= 1 && xx <= nx - 2) ? cupd : 0u;
      if (!kAux || !u)
        return 0u;
      unsigned xin = 0;
#pragma unroll
      for (int c = 0; c < 3; ++c)
        if (xx >= p.ilo[kb + c][0] && xx < p.ihi[kb + c][0])
          xin |= 3u << (2 * c);
      return ~(xin & (yz_in >> (2 * kb))) & (u * 0x15u);   // the update mask of each component's two bits
    };
    // State carried from one plane to the next.  Two sets are used in turn
    // (set P holds this plane's values, set 1 - P the previous plane's) and
    // the plane loop is unrolled by two, so nothing is copied.
    struct PlaneState
    {
      float h0[3][2];    // H0 of the plane
      float e1[3][2];    // E1 of the plane
      float im[3][2];    // 2 / (eps + eps') of E on the plane
      float h1[3][2];    // H1 of the plane before
      float e2[3][2];    // E2 of the plane before
      float xe1[3][2];   // PML: X of E after the first step on the plane
      float xh1[3][2];   // PML: X of H after the first step on the plane before
    };
    PlaneState sa = {}, sb = {};

    // STEADY: a plane from the fifth on, where every phase runs (the first
    // four fill the lag)
    auto plane = [&] (int i, auto par_c, auto steady_c, PlaneState &cur, PlaneState &prev)
                     __attribute__ ((always_inline)) -> bool {
      constexpr int P = decltype (par_c)::value;
      constexpr bool STEADY = decltype (steady_c)::value;
      const int st = i % NST2;
      const int x = xa - 2 + i;
      if (!tma::mbar_wait (bar + 8 * st, (phase >> st) & 1u))
      {
        s_abort = 1;
        atomicOr (err, 4);
      }
      phase ^= 1u << st;
      const unsigned char *stg = smem + st * L::STAGE;
      const T *sH = reinterpret_cast<const T *> (stg);
      const T *sE = reinterpret_cast<const T *> (stg + L::OFF_E);
      const float *sP = reinterpret_cast<const float *> (stg + L::OFF_P);
      const float *sA = reinterpret_cast<const float *> (stg + L::OFF_A);
      // exchange rows by plane parity: this plane's (written) and the
      // previous plane's (read).  Every set is rewritten two planes after it
      // was written, and the one barrier per plane lies between its readers
      // and that rewrite.
      float *XE1w = X + P * 2 * XN;
      const float *XE1r = X + (1 - P) * 2 * XN;
      float *XH1 = X + (4 + P * 2) * XN;
      float *XE2w = X + (8 + P * 2) * XN;
      const float *XE2r = X + (8 + (1 - P) * 2) * XN;

      // H0(x) on this row
#pragma unroll
      for (int c = 0; c < 3; ++c)
        V2<T>::ld (sH + c * HS + (w + 1) * HW + HZ + zl, cur.h0[c]);

      // ================= phase 1: E1(x) on every row, H1(x - 1) on rows 0 .. 14
      if (STEADY || i >= 1)
      {
        const unsigned u = (x >= 1 && x <= nx - 2) ? cupd : 0u;
        float hzm[2], hxm[2], eo[3][2];
        V2<T>::ld (sH + 2 * HS + w * HW + HZ + zl, hzm);
        V2<T>::ld (sH + 0 * HS + w * HW + HZ + zl, hxm);
        const float hym1 = V2<T>::ld1 (sH + 1 * HS + (w + 1) * HW + HZ + zl - 1);
        const float hxm1 = V2<T>::ld1 (sH + 0 * HS + (w + 1) * HW + HZ + zl - 1);
#pragma unroll
        for (int c = 0; c < 3; ++c)
          V2<T>::ld (sE + c * ES + w * EW + zl, eo[c]);
        if (has_eps)
        {
          float p0[2], px[2], py[2];
          lds2 (sP + w * PW + zl, p0);
          lds2 (sP + PS + w * PW + zl, px);
          lds2 (sP + (w + 1) * PW + zl, py);
          const float pz = sP[w * PW + zl + 2];
#pragma unroll
          for (int j = 0; j < 2; ++j)
          {
            cur.im[0][j] = __fdividef (2.f, p0[j] + px[j]);
            cur.im[1][j] = __fdividef (2.f, p0[j] + py[j]);
            cur.im[2][j] = __fdividef (2.f, p0[j] + (j == 0 ? p0[1] : pz));
          }
        }
        else
        {
#pragma unroll
          for (int j = 0; j < 2; ++j)
            cur.im[0][j] = cur.im[1][j] = cur.im[2][j] = 1.f;
        }
        float cu[3][2];
#pragma unroll
        for (int j = 0; j < 2; ++j)
        {
          const float hyl = j ? cur.h0[1][0] : hym1;
          const float hxl = j ? cur.h0[0][0] : hxm1;
          cu[0][j] = (cur.h0[2][j] - hzm[j]) - (cur.h0[1][j] - hyl);
          cu[1][j] = (cur.h0[0][j] - hxl) - (cur.h0[2][j] - prev.h0[2][j]);
          cu[2][j] = (cur.h0[1][j] - prev.h0[1][j]) - (cur.h0[0][j] - hxm[j]);
          if constexpr (!kZedge)
          {
#pragma unroll
            for (int c = 0; c < 3; ++c)
              cur.e1[c][j] = eo[c][j] + (S * cur.im[c][j]) * cu[c][j];
          }
        }
        if constexpr (kZedge)
        {
          const unsigned m = pmask (0, x);
#pragma unroll
          for (int c = 0; c < 3; ++c)
          {
            float xo[2] = {0.f, 0.f};
            if (c > 0)
              lds2 (sA + (c - 1) * (L::A_B / 4) + w * ZW + zl, xo);
            zedge_two (Tab, c, zl, S, u, (m >> (2 * c)) & 3u, xo, cu[c], cur.im[c], eo[c], cur.e1[c], cur.xe1[c]);
          }
        }
        else if (u != 3u)   // cells the step does not update keep their values (grid faces)
        {
#pragma unroll
          for (int j = 0; j < 2; ++j)
            if (!((u >> j) & 1u))
#pragma unroll
              for (int c = 0; c < 3; ++c)
                cur.e1[c][j] = eo[c][j];
        }
        sts2 (XE1w + 0 * XN + w * ZW + zl, cur.e1[0]);
        sts2 (XE1w + 1 * XN + w * ZW + zl, cur.e1[2]);
      }
      if ((STEADY || i >= 2) && w < NW - 1)
      {
        // H1(x - 1): E1(x - 1) in prev.e1, its y + 1 row from the previous
        // plane's exchange rows, its z + 1 cell from the next lane
        const int xh = x - 1;
        const unsigned u = (xh >= 1 && xh <= nx - 2) ? cupd : 0u;
        const float exn = __shfl_down_sync (kLanes, prev.e1[0][0], 1);
        const float eyn = __shfl_down_sync (kLanes, prev.e1[1][0], 1);
        float exy[2], ezy[2];
        lds2 (XE1r + 0 * XN + (w + 1) * ZW + zl, exy);
        lds2 (XE1r + 1 * XN + (w + 1) * ZW + zl, ezy);
        float a[3][2];
#pragma unroll
        for (int j = 0; j < 2; ++j)
        {
          const float eyz = j ? eyn : prev.e1[1][1];
          const float exz = j ? exn : prev.e1[0][1];
          a[0][j] = (eyz - prev.e1[1][j]) - (ezy[j] - prev.e1[2][j]);
          a[1][j] = (cur.e1[2][j] - prev.e1[2][j]) - (exz - prev.e1[0][j]);
          a[2][j] = (exy[j] - prev.e1[0][j]) - (cur.e1[1][j] - prev.e1[1][j]);
          if constexpr (!kZedge)
          {
#pragma unroll
            for (int c = 0; c < 3; ++c)
              cur.h1[c][j] = prev.h0[c][j] + S * a[c][j];
          }
        }
        if constexpr (kZedge)
        {
          const float one[2] = {1.f, 1.f};
          const unsigned m = pmask (3, xh);
#pragma unroll
          for (int c = 0; c < 3; ++c)
          {
            float xo[2] = {0.f, 0.f};
            if (c > 0)
              lds2 (sA + (1 + c) * (L::A_B / 4) + w * ZW + zl, xo);
            zedge_two (Tab, 3 + c, zl, S, u, (m >> (2 * c)) & 3u, xo, a[c], one, prev.h0[c], cur.h1[c], cur.xh1[c]);
          }
        }
        else if (u != 3u)
        {
#pragma unroll
          for (int j = 0; j < 2; ++j)
            if (!((u >> j) & 1u))
#pragma unroll
              for (int c = 0; c < 3; ++c)
                cur.h1[c][j] = prev.h0[c][j];
        }
        sts2 (XH1 + 0 * XN + w * ZW + zl, cur.h1[0]);
        sts2 (XH1 + 1 * XN + w * ZW + zl, cur.h1[2]);
      }

      __syncthreads ();   // E1 / H1 rows visible, stage st read
      if (s_abort)
      {
        // wait (bounded) for the copies still in flight into the other stages
        if (leader)
          for (int k = 1; k < NST2 && i + k < np; ++k)
          {
            const int so = (st + k) % NST2;
            tma::mbar_wait (bar + 8 * so, (phase >> so) & 1u);
          }
        return false;
      }
      if (leader && i + NST2 < np)
        issue (st, x + NST2, zs, Y);

      // ================= phase 2: E2(x - 1) on rows 1 .. 14, H2(x - 2) on rows 1 .. 13
      if ((STEADY || i >= 3) && w >= 1 && w < NW - 1)
      {
        const int xe = x - 1;
        const unsigned u = (xe >= 1 && xe <= nx - 2) ? cupd : 0u;
        const float hyl = __shfl_up_sync (kLanes, cur.h1[1][1], 1);
        const float hxl = __shfl_up_sync (kLanes, cur.h1[0][1], 1);
        float hzm[2], hxm[2];
        lds2 (XH1 + 1 * XN + (w - 1) * ZW + zl, hzm);
        lds2 (XH1 + 0 * XN + (w - 1) * ZW + zl, hxm);
        float cu[3][2];
#pragma unroll
        for (int j = 0; j < 2; ++j)
        {
          const float hyz = j ? cur.h1[1][0] : hyl;
          const float hxz = j ? cur.h1[0][0] : hxl;
          cu[0][j] = (cur.h1[2][j] - hzm[j]) - (cur.h1[1][j] - hyz);
          cu[1][j] = (cur.h1[0][j] - hxz) - (cur.h1[2][j] - prev.h1[2][j]);
          cu[2][j] = (cur.h1[1][j] - prev.h1[1][j]) - (cur.h1[0][j] - hxm[j]);
          if constexpr (!kZedge)
          {
#pragma unroll
            for (int c = 0; c < 3; ++c)
              cur.e2[c][j] = prev.e1[c][j] + (S * prev.im[c][j]) * cu[c][j];
          }
        }
        const bool store = own && xe >= xa && xe <= xb;
        const size_t id = (size_t) xe * sx + rowoff;
        if constexpr (kZedge)
        {
          const unsigned mE2 = pmask (0, xe);
#pragma unroll
          for (int c = 0; c < 3; ++c)
          {
            const unsigned b = (mE2 >> (2 * c)) & 3u;
            float xn[2] = {0.f, 0.f};
            zedge_two (Tab, c, zl, S, u, b, prev.xe1[c], cu[c], prev.im[c], prev.e1[c], cur.e2[c], xn);
            if (pair_along (c, 2) != 1 && b && store)
              store_aux (p.aux_new[c] + id, b, xn);
          }
        }
        else if (u != 3u)
        {
#pragma unroll
          for (int j = 0; j < 2; ++j)
            if (!((u >> j) & 1u))
#pragma unroll
              for (int c = 0; c < 3; ++c)
                cur.e2[c][j] = prev.e1[c][j];
        }
        if (store)
        {
#pragma unroll
          for (int c = 0; c < 3; ++c)
            V2<T>::st (reinterpret_cast<T *> (p.e_new[c]) + id, cur.e2[c]);
        }
        sts2 (XE2w + 0 * XN + w * ZW + zl, cur.e2[0]);
        sts2 (XE2w + 1 * XN + w * ZW + zl, cur.e2[2]);
      }
      if ((STEADY || i >= 4) && w >= 1 && w <= kTb2Yown)
      {
        const int xh = x - 2;
        const unsigned u = (xh >= 1 && xh <= nx - 2) ? cupd : 0u;
        const float exn = __shfl_down_sync (kLanes, prev.e2[0][0], 1);
        const float eyn = __shfl_down_sync (kLanes, prev.e2[1][0], 1);
        float exy[2], ezy[2];
        lds2 (XE2r + 0 * XN + (w + 1) * ZW + zl, exy);
        lds2 (XE2r + 1 * XN + (w + 1) * ZW + zl, ezy);
        float h2[3][2], a[3][2];
#pragma unroll
        for (int j = 0; j < 2; ++j)
        {
          const float eyz = j ? eyn : prev.e2[1][1];
          const float exz = j ? exn : prev.e2[0][1];
          a[0][j] = (eyz - prev.e2[1][j]) - (ezy[j] - prev.e2[2][j]);
          a[1][j] = (cur.e2[2][j] - prev.e2[2][j]) - (exz - prev.e2[0][j]);
          a[2][j] = (exy[j] - prev.e2[0][j]) - (cur.e2[1][j] - prev.e2[1][j]);
          if constexpr (!kZedge)
          {
#pragma unroll
            for (int c = 0; c < 3; ++c)
              h2[c][j] = prev.h1[c][j] + S * a[c][j];
          }
        }
        const bool store = own && xh >= xa && xh <= xb;
        const size_t id = (size_t) xh * sx + rowoff;
        if constexpr (kZedge)
        {
          const float one[2] = {1.f, 1.f};
          const unsigned mH2 = pmask (3, xh);
#pragma unroll
          for (int c = 0; c < 3; ++c)
          {
            const unsigned b = (mH2 >> (2 * c)) & 3u;
            float xn[2] = {0.f, 0.f};
            zedge_two (Tab, 3 + c, zl, S, u, b, prev.xh1[c], a[c], one, prev.h1[c], h2[c], xn);
            if (pair_along (3 + c, 2) != 1 && b && store)
              store_aux (p.aux_new[3 + c] + id, b, xn);
          }
        }
        else if (u != 3u)
        {
#pragma unroll
          for (int j = 0; j < 2; ++j)
            if (!((u >> j) & 1u))
#pragma unroll
              for (int c = 0; c < 3; ++c)
                h2[c][j] = prev.h1[c][j];
        }
        if (store)
        {
#pragma unroll
          for (int c = 0; c < 3; ++c)
            V2<T>::st (reinterpret_cast<T *> (p.h_new[c]) + id, h2[c]);
        }
      }

      return true;
    };

    using P0 = std::integral_constant<int, 0>;
    using P1 = std::integral_constant<int, 1>;
    using FILL = std::integral_constant<bool, false>;
    using RUN = std::integral_constant<bool, true>;
    int i = 0;
    for (; i < np && i < 4; i += 2)
    {
      if (!plane (i, P0{}, FILL{}, sa, sb))
      {
        aborted = true;
        break;
      }
      if (i + 1 < np && !plane (i + 1, P1{}, FILL{}, sb, sa))
      {
        aborted = true;
        break;
      }
    }
    for (; !aborted && i < np; i += 2)
    {
      if (!plane (i, P0{}, RUN{}, sa, sb))
      {
        aborted = true;
        break;
      }
      if (i + 1 < np && !plane (i + 1, P1{}, RUN{}, sb, sa))
      {
        aborted = true;
        break;
      }
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

template <typename T>
std::string plan_t (Sweep2Plan &pl, const FusedParams &p, void *const e[2][3], void *const h[2][3],
                    float *const aux[2][6], const float *eps, int sm_count)
{
  using L = L2<T>;
  const bool half = sizeof (T) == 2;
  for (int b = 0; b < 2; ++b)
  {
    Sweep2Maps &m = pl.maps[b];
    for (int c = 0; c < 3; ++c)
      if (!make_map (m.h[c], h[b][c], half, p.g.n, L::HW, L::HR) ||
          !make_map (m.e[c], e[b][c], half, p.g.n, L::EW, L::ER))
        return "tensor map encoding failed";
    if (eps)
    {
      if (!make_map (m.eps, eps, false, p.g.n, L::PW, L::PR))
        return "tensor map encoding failed";
    }
    else
      m.eps = m.e[0];   // never used
    for (int k = 0; k < 6; ++k)
    {
      if (p.use_pml && aux && aux[b][k])
      {
        if (!make_map (m.aux[k], aux[b][k], false, p.g.n, ZW, NW))
          return "tensor map encoding failed";
      }
      else
        m.aux[k] = m.e[0];   // never used
    }
  }
  int per_sm = 0;
  for (int mode = 0; mode < 3; mode += 2)
  {
    auto kern = mode == 0 ? sweep2_kernel<T, 0> : sweep2_kernel<T, 2>;
    if (cudaFuncSetAttribute (kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) L::TOTAL) != cudaSuccess)
    {
      cudaGetLastError ();
      return "shared memory request refused";
    }
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor (&n, kern, 32 * NW, L::TOTAL) != cudaSuccess || n < 1)
    {
      cudaGetLastError ();
      return "kernel does not fit on an SM";
    }
    per_sm = mode ? std::min (per_sm, n) : n;
  }
  pl.smem = L::TOTAL;
  pl.ctas = sm_count * per_sm;
  pl.work.zown = L::ZOWN;
  pl.work.zoff = L::ZOFF;
  pl.work.nzt = 1;
  // tiles until the last one's own cells reach z = nz - 2
  const int zrel = 2 * L::OHI + 2 - L::ZOFF;
  while (L::ZOWN * (pl.work.nzt - 1) + zrel < p.g.n[2] - 1)
    ++pl.work.nzt;
  return "";
}

template <typename T>
int launch_t (const Sweep2Plan &pl, int set, const FusedParams &p, int *err, cudaStream_t s, const SweepStreams &ss)
{
  const dim3 block (32, NW);
  constexpr unsigned sm = L2<T>::TOTAL;
  const bool conc = ss.side[0] && pl.items[0] > 0 && pl.items[2] > 0;
  cudaStream_t s0 = s;
  if (conc)
  {
    cudaEventRecord (ss.fork, s);
    cudaStreamWaitEvent (ss.side[0], ss.fork, 0);
    s0 = ss.side[0];
  }
  int n = 0;
  if (pl.items[2] > 0)
  {
    sweep2_kernel<T, 2><<<pl.ctas, block, sm, s>>> (pl.maps[set], p, pl.work, err);
    ++n;
  }
  if (pl.items[0] > 0)
  {
    sweep2_kernel<T, 0><<<pl.ctas, block, sm, s0>>> (pl.maps[set], p, pl.work, err);
    ++n;
  }
  if (conc)
  {
    cudaEventRecord (ss.join[0], s0);
    cudaStreamWaitEvent (s, ss.join[0], 0);
  }
  return n;
}

}  // namespace

std::string sweep2_plan (Sweep2Plan &plan, const FusedParams &p, void *const e[2][3], void *const h[2][3],
                         float *const aux[2][6], const float *eps, int sm_count, int chunk, unsigned long long *ctr,
                         int x0, int x1, int y0, int y1)
{
  const int *n = p.g.n;
  chunk = std::min (std::max (chunk, 1), kTb2MaxChunk);
  if (p.g.drop != 0)
    return "2-D grid";
  if (p.ps_mask)
    return "point source";
  if (p.use_meta)
    return "metamaterials";
  const int unit = p.fp16 ? 8 : 4;
  if (n[2] % unit != 0)
    return "nz is not a multiple of one 16-byte unit";
  if (n[0] < 3 || n[1] < 3 || n[2] < 3)
    return "grid too small";
  if (x1 < 0)
    x1 = n[0] - 1;
  if (y1 < 0)
    y1 = n[1] - 1;
  if (x0 < 1 || x1 > n[0] - 1 || x0 >= x1 || y0 < 1 || y1 > n[1] - 1 || y0 >= y1)
    return "bad owned range";
  std::string why = p.fp16 ? plan_t<__half> (plan, p, e, h, aux, eps, sm_count)
                           : plan_t<float> (plan, p, e, h, aux, eps, sm_count);
  if (!why.empty ())
    return why;
  Sweep2Work &w = plan.work;
  w.yoff = y0 - 1;
  w.yend = y1;
  w.nyt = (y1 - y0 + kTb2Yown - 1) / kTb2Yown;
  // x chunks of about `chunk` planes over the owned planes x0 .. x1 - 1;
  // with PML, the planes where every component is PML-free (with the two
  // halo planes) form their own segment, so that no chunk mixes them
  std::vector<int> seg = {x0};
  if (p.use_pml)
  {
    int lo = 1, hi = n[0] - 2;
    for (int k = 0; k < 6; ++k)
    {
      lo = std::max (lo, p.ilo[k][0] + 2);
      hi = std::min (hi, p.ihi[k][0] - 3);
    }
    if (lo > x0 && lo < x1 && lo <= hi)
      seg.push_back (lo);
    if (hi + 1 > x0 && hi + 1 < x1 && lo <= hi)
      seg.push_back (hi + 1);
  }
  seg.push_back (x1);
  w.nch = 0;
  w.xcut[0] = x0;
  for (size_t sg = 0; sg + 1 < seg.size (); ++sg)
  {
    const int len = seg[sg + 1] - seg[sg];
    int m = std::max (1, (len + chunk - 1) / chunk);
    m = std::min (m, kMaxChunks - w.nch);
    for (int j = 1; j <= m; ++j)
      w.xcut[++w.nch] = seg[sg] + (int) ((long long) len * j / m);
  }
  for (int j = 0; j < w.nch; ++j)
    if (w.xcut[j + 1] - w.xcut[j] > kTb2MaxChunk)
      return "grid too long in x for the chunk count";
  w.nitems = w.nzt * w.nyt * w.nch;
  w.ctr = ctr;
  plan.items[0] = plan.items[1] = plan.items[2] = 0;
  for (int it = 0; it < w.nitems; ++it)
    ++plan.items[sweep2_item_class (p, w, it)];
  if (plan.items[1] > 0)
    return "x / y PML cells in the two-step region (the single-step shell takes them)";
  if (plan.ctas > w.nitems)
    plan.ctas = w.nitems;
  return "";
}

int launch_sweep2 (const Sweep2Plan &plan, int set, const FusedParams &p, int *err, cudaStream_t s,
                   const SweepStreams &ss)
{
  return p.fp16 ? launch_t<__half> (plan, set, p, err, s, ss) : launch_t<float> (plan, set, p, err, s, ss);
}

}  // namespace fdtdb
