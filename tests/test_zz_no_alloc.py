"""The allocation-free reduction entry point against the allocating one.

fdtd_reduce_sq_noalloc exists for callers that must not allocate device
memory while they run (an application whose own allocator owns the device's
memory budget, or a real-time loop where cudaMalloc can stall and cudaFree
synchronises the device).  It keeps its per-block partial sums in one static
device array instead of allocating scratch.  This test calls it through the C
ABI on field data the library produced, twice in a row with different inputs,
and compares each result with fdtd_reduce, the existing entry point that uses
the context's allocated scratch.  Tolerance: 1e-12 relative, because the two
entry points sum the same values with different block partitions.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bind(lib):
    fn = lib.fdtd_reduce_sq_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_int,
                   ctypes.c_double, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return fn


def test_noalloc_reduction_matches_allocating_reduction(fdtd):
    import torch

    lib = fdtd.load_library()
    noalloc = _bind(lib)
    kw = dict(mode=3, size=(24, 22, 26), use_pml=True, pml=4, use_tfsf=True, tfsf_left=7, tfsf_right=7,
              teta=30, phi=45, psi=0, precision=fdtd.PREC_FP32)
    with fdtd.Simulation(device=0, **kw) as sim:
        sim.step(30)
        sim.sync()
        l2 = sim.reduce(fdtd.REDUCE_L2)
        torch.cuda.set_device(0)
        buf = torch.empty(sim.cells, dtype=torch.float64, device="cuda:0")
        out = torch.zeros(1, dtype=torch.float64, device="cuda:0")
        for comp in ("Ey", "Hx"):   # two calls in a row, different inputs
            k = fdtd.COMPONENTS.index(comp)
            sim.field_device(comp, buf.data_ptr())
            sim.sync()
            out.fill_(-1.0)
            torch.cuda.synchronize()
            st = noalloc(buf.data_ptr(), 0, sim.cells, None, 0, 1.0, 0, out.data_ptr(), None)
            assert st == 0, lib.fdtd_last_error()
            torch.cuda.synchronize()
            got = float(out.item())
            ref = float(l2[k])
            assert ref > 0
            assert abs(got - ref) <= 1e-12 * ref, (comp, got, ref)
        # an explicit block count within the static array gives the same sum
        st = noalloc(buf.data_ptr(), 0, sim.cells, None, 0, 1.0, 7, out.data_ptr(), None)
        assert st == 0
        torch.cuda.synchronize()
        assert abs(float(out.item()) - float(l2[3])) <= 1e-12 * float(l2[3])
        # more partials than the static array holds is refused, nothing is launched
        assert noalloc(buf.data_ptr(), 0, sim.cells, None, 0, 1.0, 1025, out.data_ptr(), None) == -1
