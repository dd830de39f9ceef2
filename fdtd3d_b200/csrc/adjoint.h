// adjoint.h - reverse-mode (adjoint) differentiation of the 2-D TMz step.
//
// The forward model is the library's FP32 TMz step (fast_kernels.cu: H
// stored as eta0*H, interior cells F += S/m * curl, PML cells through the
// auxiliary X), evaluated here in FP32 or FP64.  The objective is
//   J = sum over t = 1 .. steps of sum over the probe box of Ez_t^2
// (Ez_t after the E half-step and E point source of step t), accumulated in
// FP64 with compensation.  The gradient is dJ/d(eps) for every cell, the
// exact transpose of the discrete step (PML included), obtained by
// checkpointing the state every K steps and recomputing one segment at a
// time in the reverse sweep.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "setup.h"

namespace fdtdb {

// Device memory kept between runs of one context: a run takes it when it is
// large enough and replaces it otherwise (freed by the owner).
struct AdjointCache
{
  void *base = nullptr;
  size_t bytes = 0;
};

struct AdjointRun
{
  uint32_t steps = 0;
  uint32_t every = 0;          // checkpoint interval K
  int probe_lo[2] = {0, 0};
  int probe_hi[2] = {0, 0};    // exclusive
  bool fp64 = false;
  AdjointCache *cache = nullptr;   // null: allocate and free per run
  long long wait_limit_ns = 0;     // time limit of one grid-barrier wait (<= 0: 2 s)
};

// eps_dev: per-cell permittivity on the device (float when eps_is_double is
// false), nx * ny values in the library's layout (x outer, y inner).
// objective: host double.  grad_host: nx * ny doubles (host) or null for a
// forward-only run.  Returns "" or an error message.
std::string adjoint_run (const Geometry &g, const void *eps_dev, bool eps_is_double, const AdjointRun &run,
                         double *objective, double *grad_host, int sm_count, cudaStream_t s);

}  // namespace fdtdb
