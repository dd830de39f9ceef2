// incident_dev.cuh - incident-wave value at a cell for the TF/SF
// corrections of the FP32 / FP16-storage kernels.
#pragma once

#include "params.h"

namespace fdtdb {

// Incident value of component k at integer cell (px, py, pz): the position
// of the component (cell + its min_fp offset) projected on the wave vector,
// linear interpolation in the 1-D incident grid, times the component's
// projection (InternalScheme.inc.h:1386-1835 approximateIncidentWave*).
// Sets *err = 1 and returns 0 when the position falls outside the grid.
__device__ __forceinline__ double inc_at (const GeomDev &g, const double *inc, int inc_len, int *err, int k, int px,
                                          int py, int pz)
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

}  // namespace fdtdb
