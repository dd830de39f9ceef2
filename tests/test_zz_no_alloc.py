"""The allocation-free reduction entry point against the allocating one.

fdtd_reduce_sq_noalloc exists for callers that must not allocate device
memory while they run (an application whose own allocator owns the device's
memory budget, or a real-time loop where cudaMalloc can stall and cudaFree
synchronises the device).  It keeps its per-block partial sums in one static
device array instead of allocating scratch.  These tests call it through the
C ABI on field data the library produced:

* twice in a row with different inputs, each result compared with
  fdtd_reduce, the existing entry point that uses the context's allocated
  scratch;
* for every source kind (double, float, half) and weight kind (none, float,
  double), with scale 2.5, on a side stream, against a torch float64 sum of
  weight * x^2 * scale of the same values.

Tolerance: 1e-12 relative, because the entry points sum the same values with
different block partitions (all sums are compensated FP64).
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


KW = dict(mode=3, size=(24, 22, 26), use_pml=True, pml=4, use_tfsf=True, tfsf_left=7, tfsf_right=7,
          teta=30, phi=45, psi=0)


def test_noalloc_reduction_matches_allocating_reduction(fdtd):
    import torch

    lib = fdtd.load_library()
    noalloc = _bind(lib)
    with fdtd.Simulation(device=0, precision=fdtd.PREC_FP32, **KW) as sim:
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
        assert b"1024" in lib.fdtd_last_error()
        # an unknown weight kind is refused (kinds: 0 none, 1 float, 2 double)
        assert noalloc(buf.data_ptr(), 0, sim.cells, buf.data_ptr(), 3, 1.0, 0, out.data_ptr(), None) == -1
        assert b"weight_kind" in lib.fdtd_last_error()


@pytest.mark.parametrize("src_kind", [0, 1, 2])
@pytest.mark.parametrize("weight_kind", [0, 1, 2])
def test_noalloc_kinds_weights_scale_stream(fdtd, src_kind, weight_kind):
    import torch

    lib = fdtd.load_library()
    noalloc = _bind(lib)
    torch.cuda.set_device(0)
    with fdtd.Simulation(device=0, precision=fdtd.PREC_FP32, **KW) as sim:
        sim.step(30)
        sim.sync()
        field = torch.empty(sim.cells, dtype=torch.float64, device="cuda:0")
        sim.field_device("Ey", field.data_ptr())
        sim.sync()
    torch.cuda.synchronize()
    src = {0: field, 1: field.float(), 2: field.half()}[src_kind].contiguous()
    gen = torch.Generator(device="cpu").manual_seed(11 + 3 * src_kind + weight_kind)
    wv = torch.rand(src.numel(), generator=gen, dtype=torch.float64) + 0.5
    weight = None
    if weight_kind == 1:
        weight = wv.float().cuda()
    elif weight_kind == 2:
        weight = wv.cuda()
    scale = 2.5
    x = src.double()
    ref = (x * x * scale) if weight is None else (weight.double() * x * x * scale)
    ref = float(ref.sum().item())
    assert ref > 0
    side = torch.cuda.Stream()
    outs = []
    for _ in range(2):   # two calls in a row on the side stream
        out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda:0")
        torch.cuda.synchronize()
        st = noalloc(src.data_ptr(), src_kind, src.numel(), None if weight is None else weight.data_ptr(),
                     weight_kind, scale, 0, out.data_ptr(), side.cuda_stream)
        assert st == 0, lib.fdtd_last_error()
        side.synchronize()
        outs.append(float(out.item()))
    for got in outs:
        assert abs(got - ref) <= 1e-12 * ref, (src_kind, weight_kind, got, ref)
