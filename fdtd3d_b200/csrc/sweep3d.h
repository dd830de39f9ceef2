// sweep3d.h - TMA-pipelined one-sweep E+H step for the 3-D FP32 and
// FP16-storage forms (uniform mu, no metamaterials, nz a multiple of one
// 16-byte unit).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "fused3d.h"

namespace fdtdb {

// Tensor-map descriptors of one "old" buffer set.  H boxes carry a one-row
// halo in y and one 16-byte halo on both sides in z; E, eps and PML
// auxiliary boxes start at the tile origin.
struct SweepMaps
{
  CUtensorMap h[3];
  CUtensorMap e[3];
  CUtensorMap eps;
  CUtensorMap aux[6];
  CUtensorMap auxn[6];         // narrow (32-cell) boxes for planes whose PML cells are all at a z edge
};

// Tiled 3-D tensor map over an (n[0], n[1], n[2]) array (z fastest, FP32 or
// FP16), box bw (z) x bh (y) x 1 (x), 64-byte L2 promotion, zero fill.
bool make_map (CUtensorMap &m, const void *base, bool half, const int n[3], int bw, int bh);

constexpr int kMaxChunks = 256;   // x chunks per step (the chunk grows for larger grids)

struct SweepWork
{
  int nzt, nyt, nch, nitems, chunk;
  int xcut[kMaxChunks + 4];    // chunk c covers planes xcut[c] .. xcut[c + 1] - 1
  int lean;                    // 0: every item goes to the full class
  unsigned long long *ctr;     // per item class c: [2c] next item, [2c + 1] CTAs finished; the last
                               // CTA of a launch resets both
  const int *list;             // device list of the items to run (null: items 0 .. nitems - 1)
  int nlist;                   // its length
};

struct SweepPlan
{
  int wy = 0;                  // warps per CTA, one y row each (last row = ring)
  int ctas = 0;                // persistent CTAs
  unsigned smem = 0;           // dynamic shared memory per CTA
  int items[4] = {0, 0, 0, 0}; // items per class: lean, z-edge PML, full, PML
  SweepWork work{};
  SweepMaps maps[2];           // maps[b]: buffer set b as the old set
};

// Tiles per axis, x chunks (cut at the PML edges, at most `chunk` planes
// each) and items for a given CTA height.
void sweep3d_items (const FusedParams &p, int wy, int chunk, SweepWork &w);

// Builds the tensor maps and launch shape.  e/h[b][c] are the field buffers
// of set b, aux[b][k] the PML auxiliaries of set b (null without PML), eps
// the FP32 permittivity (or null).  Returns "" or the reason the kernel
// cannot serve this geometry.
std::string sweep3d_plan (SweepPlan &plan, const FusedParams &p, void *const e[2][3], void *const h[2][3],
                          float *const aux[2][6], const float *eps, int sm_count, int wy, int chunk,
                          unsigned long long *ctr, bool lean = true);

// A plan that runs only some items: x chunks cut at `cuts` (increasing, from
// 1 to nx - 1), and the items of `host_list` (ids over the z tile, y tile and
// x chunk grid of those cuts), copied to the device array `dev_list` (at least
// host_list.size () ints, owned by the caller).  Used for the PML shell of the
// two-step scheme.
std::string sweep3d_plan_list (SweepPlan &plan, const FusedParams &p, void *const e[2][3], void *const h[2][3],
                               float *const aux[2][6], const float *eps, int sm_count, const std::vector<int> &cuts,
                               const std::vector<int> &host_list, int *dev_list, unsigned long long *ctr,
                               cudaStream_t s);

// Tiles of the single-step sweep (8-warp CTAs): z tile zt owns z cells
// 128 zt .. 128 zt + 127, y tile yt rows 1 + 7 yt .. 7 + 7 yt.
constexpr int kSweepTileZ = 128;
constexpr int kSweepTileY = 7;

// Side streams for the item classes: the classes of one step write disjoint
// items and read only the old set, so they may run concurrently; then the
// SMs that one class's persistent CTAs leave take the next class's CTAs
// instead of idling through its tail.  fork is recorded on the main stream,
// join[j] on side[j] (all null: one stream).
struct SweepStreams
{
  cudaStream_t side[2] = {nullptr, nullptr};
  cudaEvent_t fork = nullptr, join[2] = {nullptr, nullptr};
};

// One time step with buffer set `set` as the old set (one launch per item
// class that has items; returns how many).  With side streams the z-edge
// and the lean class run on them, joined back into s before returning.
int launch_sweep3d (const SweepPlan &plan, int set, const FusedParams &p, int *err, cudaStream_t s,
                    const SweepStreams &ss = SweepStreams ());

}  // namespace fdtdb

namespace fdtdb {

// TF/SF post pass of the sweep: the cells within one cell of a TF/SF face
// as disjoint boxes.  Every TF/SF term covers a box whole or misses it, so
// the terms that act on a box are one mask per component.
struct BandBox
{
  int lo[3], hi[3];            // cells lo .. hi - 1 per axis
  unsigned mask;               // bit 4k + t: term t of component k (Ex..Hz) covers the box
  unsigned nmask[3];           // the same for Ex..Ez over the box moved by +1 along x, y, z
};

struct TfsfBand
{
  int nbox = 0;
  long long cells = 0;
  BandBox *boxes = nullptr;    // device array
  int nblk = 0;                // CTAs of the post pass
  int2 *blk = nullptr;         // per CTA: the box and the first of its cells the CTA takes
};

// Host part: the band's boxes from the TF/SF terms (E terms and their
// -x/-y/-z neighbours, H terms) with their term masks, and the CTA table.
// Returns "" when the post pass can serve the geometry (no band cell is a
// PML cell of any component), else the reason.
std::string tfsf_band_boxes (const FusedParams &p, std::vector<BandBox> &boxes, std::vector<int2> &blk);

// Adds the TF/SF corrections to the new E and H buffers after a sweep step
// that ran with tfsf_post = 1 (one launch; returns how many).
int launch_tfsf_post (const TfsfBand &band, const FusedParams &p, int *err, cudaStream_t s);

}  // namespace fdtdb
