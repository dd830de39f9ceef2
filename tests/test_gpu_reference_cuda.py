"""The reference's own CUDA path beside this library's FP64 plain form, on the same B200.

`oracle/_ref/fdtd3d_cuda` is the unmodified reference built with CUDA_ENABLED
for sm_100a by `oracle/Makefile` (target ref_cuda): its one-thread-per-cell
FP64 kernels, about 40 launches per time step
(Source/Scheme/InternalScheme.inc.h:21-432, launches 877-1146), driven by its
own `--use-cuda` step loop.  Run with the launch shape of the reference's
own GPU tests (`--num-cuda-threads x:4,y:4,z:4`, Tests/suite/*/run.sh).

* Config 1 (3-D 80^3, PML 10, TF/SF 15, theta = phi = psi = 0, 100 steps):
  every field of the reference's GPU run against this library's FP64 plain
  form (which is bit-identical to the reference CPU build).  nvcc contracts
  the reference's multiply-adds into FMAs (its CMake passes no --fmad=false),
  so the two agree to rounding, not bit for bit: relative L2 <= 1e-12 per
  field family, the bar of the FP64 drop-in.
* Both runs are timed by wall clock around the step loop (the reference's own
  'Total time' line, and fdtd_step + fdtd_sync here), on config 1 and on a
  larger oblique-incidence grid (200^3, PML 16, TF/SF 32, theta 30, phi 45,
  60 steps), and the rates are printed.
"""
import os
import time

import numpy as np
import pytest

from oracle.oracle import REF_CUDA_BIN, run_reference

pytestmark = pytest.mark.gpu

CUDA_ARGS = ["--use-cuda", "--cuda-gpus", "0", "--num-cuda-threads", "x:4,y:4,z:4"]
CONFIG1 = dict(mode=3, size=80, use_pml=True, pml=10, use_tfsf=True, tfsf_left=15, tfsf_right=15,
               teta=0.0, phi=0.0, psi=0.0, dx=0.0005, wavelength=0.02, courant=0.5)
LARGE = dict(mode=3, size=200, use_pml=True, pml=16, use_tfsf=True, tfsf_left=32, tfsf_right=32,
             teta=30.0, phi=45.0, psi=0.0, dx=0.0005, wavelength=0.02, courant=0.5)


def _need_binary():
    if not os.path.exists(REF_CUDA_BIN):
        pytest.skip("oracle/_ref/fdtd3d_cuda is not built (make -C oracle ref_cuda REF_ROOT=...)")


def _ours(fdtd, kw, steps):
    with fdtd.Simulation(precision=fdtd.PREC_FP64_PLAIN, **kw) as sim:
        sim.step(1)   # t = 0: no field update, sets up the step tables
        sim.sync()
        t0 = time.perf_counter()
        sim.step(steps - 1, t_start=1)
        sim.sync()
        dt = time.perf_counter() - t0
        fields = {c: sim.field(c).copy() for c in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")}
    return fields, dt


def test_reference_cuda_config1_matches_and_is_timed(fdtd):
    _need_binary()
    steps = 100
    ref, t_ref = run_reference(binary=REF_CUDA_BIN, extra_args=CUDA_ARGS, steps=steps, timeout=900, **CONFIG1)
    ours, t_ours = _ours(fdtd, CONFIG1, steps)
    for fam in (("Ex", "Ey", "Ez"), ("Hx", "Hy", "Hz")):
        r = np.concatenate([ref[c].ravel() for c in fam])
        g = np.concatenate([ours[c].ravel() for c in fam])
        err = np.linalg.norm(g - r) / np.linalg.norm(r)
        print(f"config 1 {fam[0][0]} family: relative L2 reference CUDA vs FP64 plain form {err:.3e}")
        assert err <= 1e-12, (fam, err)
    cells = 80 ** 3 * (steps - 1)   # the reference skips the field update at t = 0
    print(f"config 1: reference CUDA {cells / t_ref / 1e9:.4f} Gcell-updates/s ({t_ref:.3f} s), "
          f"FP64 plain form {cells / t_ours / 1e9:.4f} Gcell-updates/s ({t_ours:.3f} s), "
          f"ratio {t_ref / t_ours:.1f}")


def test_reference_cuda_larger_grid_timed(fdtd):
    _need_binary()
    steps = 60
    _, t_ref = run_reference(binary=REF_CUDA_BIN, extra_args=CUDA_ARGS, steps=steps, save=False, timeout=900,
                             **LARGE)
    _, t_ours = _ours(fdtd, LARGE, steps)
    cells = 200 ** 3 * (steps - 1)
    print(f"200^3 oblique: reference CUDA {cells / t_ref / 1e9:.4f} Gcell-updates/s ({t_ref:.3f} s), "
          f"FP64 plain form {cells / t_ours / 1e9:.4f} Gcell-updates/s ({t_ours:.3f} s), "
          f"ratio {t_ref / t_ours:.1f}")
    assert t_ref > 0 and t_ours > 0
