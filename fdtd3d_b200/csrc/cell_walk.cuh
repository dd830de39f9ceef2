// cell_walk.cuh - the grid-stride loop of the per-cell kernels over the
// interior box (ix x iy x iz cells, z fastest).
//
// A thread's first cell index is decomposed into (x, y, z) once; every later
// cell adds the stride's own decomposition, with at most one wrap per axis
// (each remainder is below its extent).  This replaces three 64-bit
// divisions per cell, which otherwise dominate the instruction count of the
// per-cell kernels.
#pragma once

#include <cstdint>

namespace fdtdb {

struct CellWalk
{
  int64_t tid, total, stride;
  int cx, cy, cz;   // cell offsets inside the box
  int sx, sy, sz;   // the stride's decomposition
  int iy, iz;

  __device__ CellWalk (int64_t start, int64_t step, int ix, int iy_, int iz_)
      : tid (start), total ((int64_t) ix * iy_ * iz_), stride (step), iy (iy_), iz (iz_)
  {
    const int64_t plane = (int64_t) iy_ * iz_;
    cz = (int) (start % iz_);
    cy = (int) ((start / iz_) % iy_);
    cx = (int) (start / plane);
    sz = (int) (step % iz_);
    sy = (int) ((step / iz_) % iy_);
    sx = (int) (step / plane);
  }
  __device__ bool ok () const { return tid < total; }
  __device__ void next ()
  {
    tid += stride;
    cz += sz;
    int c = cz >= iz;
    cz -= c ? iz : 0;
    cy += sy + c;
    c = cy >= iy;
    cy -= c ? iy : 0;
    cx += sx + c;
  }
};

}  // namespace fdtdb
