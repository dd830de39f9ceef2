// sweep2.h - two time steps per pass over HBM (temporal blocking) for the
// 3-D FP32 / FP16-storage one-sweep step.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <string>

#include "fused3d.h"
#include "sweep3d.h"

namespace fdtdb {

// Tile of the two-step kernel: 16 warps, one row each (rows Y .. Y + 15),
// 2 z cells per lane (z = zs .. zs + 63).  Rows Y + 1 .. Y + 13 and the
// cells of the middle 60 (FP32) or 56 (FP16 storage) z columns are the
// tile's own; the rest is the halo whose first-step values the second step
// needs (recomputed, never exchanged).
constexpr int kTb2Warps = 16;
constexpr int kTb2Zw = 64;
constexpr int kTb2Yown = 13;
constexpr int kTb2MaxChunk = 256;  // x planes per item at most
// x planes per item by default: each item pays a four-plane pipeline fill,
// so longer items do less redundant work while a 512^3 grid still gives
// every SM several items
constexpr int kTb2Chunk = 128;

struct Sweep2Maps
{
  CUtensorMap h[3];            // box (zs - 4 .. zs + 63) x (Y - 1 .. Y + 15)
  CUtensorMap e[3];            // box (zs .. zs + 63) x (Y .. Y + 15)
  CUtensorMap eps;             // box (zs .. zs + 67) x (Y .. Y + 16)
  CUtensorMap aux[6];          // PML auxiliaries (float), box (zs .. zs + 63) x (Y .. Y + 15)
};

struct Sweep2Work
{
  int nzt, nyt, nch, nitems;
  int zown, zoff;              // z tile k's warp rows start at zown k - zoff
  int yoff;                    // y tile k's warp rows start at yoff + 13 k (own rows from yoff + 13 k + 1)
  int yend;                    // rows >= yend are not stored (the end of the rows the plan owns)
  int xcut[kMaxChunks + 4];    // chunk c owns planes xcut[c] .. xcut[c + 1] - 1
  unsigned long long *ctr;     // per item class c (3): [2c] next item, [2c + 1] CTAs finished (the last resets both)
};

// Class of item `item`: 0 (lean) when no updated cell whose first-step value
// reaches the item's own cells (planes xa - 2 .. xb + 2, rows Y .. the own
// rows' end + 2, z cells zs .. zs + 63) is a PML cell of any component; 2 (z
// edge) when those cells are PML cells only along z (x and y interior for
// every component); else 1 (PML).  Shared by the host and the kernels.
__host__ __device__ inline int sweep2_item_class (const FusedParams &p, const Sweep2Work &wk, int item)
{
  if (!p.use_pml)
    return 0;
  const int zt = item % wk.nzt;
  const int yt = (item / wk.nzt) % wk.nyt;
  const int ch = item / (wk.nzt * wk.nyt);
  const int zs = wk.zown * zt - wk.zoff, Y = wk.yoff + kTb2Yown * yt;
  const int yhi = Y + kTb2Warps - 1 < wk.yend + 1 ? Y + kTb2Warps - 1 : wk.yend + 1;
  const int lo[3] = {wk.xcut[ch] - 2, Y, zs};
  const int hi[3] = {wk.xcut[ch + 1] + 1, yhi, zs + kTb2Zw - 1};   // inclusive
  bool zpml = false;
  for (int k = 0; k < 6; ++k)
    for (int a = 0; a < 3; ++a)
    {
      const int l = lo[a] > 1 ? lo[a] : 1;
      const int h = hi[a] < p.g.n[a] - 2 ? hi[a] : p.g.n[a] - 2;
      if (l <= h && (l < p.ilo[k][a] || h >= p.ihi[k][a]))
      {
        if (a < 2)
          return 1;
        zpml = true;
      }
    }
  return zpml ? 2 : 0;
}

struct Sweep2Plan
{
  int ctas = 0;
  unsigned smem = 0;
  int items[3] = {0, 0, 0};    // items per class: lean, PML, z edge
  Sweep2Work work{};
  Sweep2Maps maps[2];          // maps[b]: buffer set b as the old set
};

// Builds the plan, or returns why the two-step kernel cannot serve the
// geometry (it serves grids without point sources or Drude media, with
// uniform mu; PML anywhere).  The kernel applies no TF/SF correction: with
// TF/SF the caller adds the pair's corrections afterwards (tfsf2.h).  The plan owns the cells of rows
// y0 .. y1 - 1 and planes x0 .. x1 - 1 (all z); y0 = 1, y1 = ny - 1,
// x0 = 1, x1 = nx - 1 is the whole grid.
std::string sweep2_plan (Sweep2Plan &plan, const FusedParams &p, void *const e[2][3], void *const h[2][3],
                         float *const aux[2][6], const float *eps, int sm_count, int chunk, unsigned long long *ctr,
                         int x0 = 1, int x1 = -1, int y0 = 1, int y1 = -1);

// Two time steps: buffer set `set` holds time t on entry; the kernel writes
// time t + 2 into set 1 - set (one launch per item class that has items;
// with side streams the lean class runs on side[0], joined back into s).
// Returns the number of launches.
int launch_sweep2 (const Sweep2Plan &plan, int set, const FusedParams &p, int *err, cudaStream_t s,
                   const SweepStreams &ss = SweepStreams ());

}  // namespace fdtdb
