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
constexpr int kTb2MaxChunk = 64;   // x planes per item (the PML class stages an x table of chunk + 4)

struct Sweep2Maps
{
  CUtensorMap h[3];            // box (zs - 4 .. zs + 63) x (Y - 1 .. Y + 15)
  CUtensorMap e[3];            // box (zs .. zs + 63) x (Y .. Y + 15)
  CUtensorMap eps;             // box (zs .. zs + 67) x (Y .. Y + 16)
};

struct Sweep2Work
{
  int nzt, nyt, nch, nitems;
  int zown, zoff;              // z tile k's warp rows start at zown k - zoff
  int xcut[kMaxChunks + 4];    // chunk c owns planes xcut[c] .. xcut[c + 1] - 1
  unsigned long long *ctr;     // per item class c: [2c] next item, [2c + 1] CTAs finished (the last resets both)
};

// Class of item `item`: 0 (lean) when no updated cell of its extended region
// (planes xa - 2 .. xb + 2, rows Y .. Y + 15, z cells zs .. zs + 63) is a
// PML cell of any component, else 1 (PML).  Shared by the host and the
// kernels.
__host__ __device__ inline int sweep2_item_class (const FusedParams &p, const Sweep2Work &wk, int item)
{
  if (!p.use_pml)
    return 0;
  const int zt = item % wk.nzt;
  const int yt = (item / wk.nzt) % wk.nyt;
  const int ch = item / (wk.nzt * wk.nyt);
  const int zs = wk.zown * zt - wk.zoff, Y = kTb2Yown * yt;
  const int lo[3] = {wk.xcut[ch] - 2, Y, zs};
  const int hi[3] = {wk.xcut[ch + 1] + 1, Y + kTb2Warps - 1, zs + kTb2Zw - 1};   // inclusive
  for (int k = 0; k < 6; ++k)
    for (int a = 0; a < 3; ++a)
    {
      const int l = lo[a] > 1 ? lo[a] : 1;
      const int h = hi[a] < p.g.n[a] - 2 ? hi[a] : p.g.n[a] - 2;
      if (l <= h && (l < p.ilo[k][a] || h >= p.ihi[k][a]))
        return 1;
    }
  return 0;
}

struct Sweep2Plan
{
  int ctas = 0;
  unsigned smem = 0;
  int items[2] = {0, 0};       // items per class: lean, PML
  Sweep2Work work{};
  Sweep2Maps maps[2];          // maps[b]: buffer set b as the old set
};

// Builds the plan, or returns why the two-step kernel cannot serve the
// geometry (it serves grids without TF/SF, point sources or Drude media,
// with uniform mu; PML anywhere).
std::string sweep2_plan (Sweep2Plan &plan, const FusedParams &p, void *const e[2][3], void *const h[2][3],
                         const float *eps, int sm_count, int chunk, unsigned long long *ctr);

// Two time steps: buffer set `set` holds time t on entry; the kernel writes
// time t + 2 into set 1 - set (one launch per item class that has items;
// with side streams the lean class runs on side[0], joined back into s).
// Returns the number of launches.
int launch_sweep2 (const Sweep2Plan &plan, int set, const FusedParams &p, int *err, cudaStream_t s,
                   const SweepStreams &ss = SweepStreams ());

}  // namespace fdtdb
