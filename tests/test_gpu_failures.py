"""Failure detection without a GPU fault.

The reference exits on every CUDA error (Source/Helpers/CudaInclude.h:41-47);
here every failure is a status code, and these tests make each kind happen
on purpose, in forms that fault, trap and hang nothing:

* a device-side wait that runs out: the grid barriers of the batch kernel and
  of the adjoint kernel take a time limit from the host; with a limit of 1 ns
  the waiting CTAs give up at their first check, raise the device error flag
  and every CTA leaves the launch.  The call reports FDTD_ERR_DEVICE, and a
  fresh batch (or the same context with the default limit) then steps
  correctly.  (The 3-D sweep's TMA pipeline waits keep their fixed limit;
  they are not forced to run out on a GPU.)
* a NaN or an infinity in a host material array: refused before anything the
  step reads changes.
* an allocation failure, injected on the host at every allocation in turn:
  the call that needed it reports FDTD_ERR_NOMEM and device memory returns to
  where it was (nothing leaked).
"""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ERR_ARG, ERR_NOMEM, ERR_DEVICE = -1, -3, -7

PHYS = dict(use_pml=True, pml=6, dx=0.0005, wavelength=0.02, courant=0.5, teta=90, phi=0, psi=90,
            point_source_mask=1 << 2, point_source_kind=1, point_source_bandwidth=0.5)


def rel_l2(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def test_batch_barrier_runs_out_then_fresh_batch_steps(fdtd):
    sizes = [(48, 40), (64, 72), (30, 90), (100, 52)]
    t0 = time.perf_counter()
    with fdtd.Batch(sizes, **PHYS) as b:
        b.set_wait_limit(1)
        b.step(40)
        with pytest.raises(fdtd.FdtdError) as e:
            b.sync()
        assert e.value.status == ERR_DEVICE, e.value
        assert "barrier" in str(e.value)
    assert time.perf_counter() - t0 < 60.0
    # a fresh batch with the default limit steps like single-instance runs
    with fdtd.Batch(sizes, **PHYS) as b:
        b.step(30)
        b.sync()
        for i, (nx, ny) in enumerate(sizes):
            with fdtd.Simulation(mode=2, size=(nx, ny), point_source=(nx // 2, ny // 2), precision=fdtd.PREC_FP32,
                                 **PHYS) as s:
                s.step(30)
                assert rel_l2(b.field(i, "Ez"), s.field("Ez")) <= 1e-6


def test_adjoint_barrier_runs_out_then_context_recovers(fdtd):
    n = 64
    kw = dict(mode=2, size=(n, n), point_source=(20, 32, 0), precision=fdtd.PREC_FP32, **PHYS)
    p0, p1 = (40, 28), (48, 36)
    with fdtd.Simulation(**kw) as ref:
        want = ref.objective(200, p0, p1, fdtd.PREC_FP32)
    assert want > 0
    with fdtd.Simulation(**kw) as sim:
        sim.set_wait_limit(1)
        t0 = time.perf_counter()
        with pytest.raises(fdtd.FdtdError) as e:
            sim.objective(200, p0, p1, fdtd.PREC_FP32)
        assert e.value.status == ERR_DEVICE, e.value
        assert "timed out" in str(e.value)
        with pytest.raises(fdtd.FdtdError) as e:
            sim.backward(200, 50, p0, p1, fdtd.PREC_FP32)
        assert e.value.status == ERR_DEVICE, e.value
        assert time.perf_counter() - t0 < 60.0
        sim.set_wait_limit(0)   # the default again: the next call starts afresh
        got = sim.objective(200, p0, p1, fdtd.PREC_FP32)
        assert got == want
        # the context's own stepping is untouched
        sim.step(20)
        sim.sync()
        assert np.isfinite(sim.field("Ez")).all()


@pytest.mark.parametrize("prec", ["PREC_FP64_PLAIN", "PREC_FP32"])
@pytest.mark.parametrize("bad", [np.nan, np.inf, -np.inf])
def test_nonfinite_material_is_refused(fdtd, prec, bad):
    kw = dict(mode=3, size=(20, 18, 24), use_pml=True, pml=4, use_tfsf=True, tfsf_left=6, tfsf_right=6,
              teta=30, phi=45, psi=0, precision=getattr(fdtd, prec))
    eps = np.full((20, 18, 24), 2.0)
    eps.reshape(-1)[4321] = bad
    with fdtd.Simulation(**kw) as sim, fdtd.Simulation(**kw) as ref:
        with pytest.raises(fdtd.FdtdError) as e:
            sim.set_material("eps", eps)
        assert e.value.status == ERR_ARG
        assert "non-finite" in str(e.value) and "4321" in str(e.value)
        # nothing changed: the refused context steps like one that never saw it
        sim.step(25)
        ref.step(25)
        for c in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
            assert np.array_equal(sim.field(c), ref.field(c)), c


def _free_bytes():
    import torch

    torch.cuda.synchronize()
    return torch.cuda.mem_get_info(0)[0]


@pytest.mark.parametrize("prec", ["PREC_FP64_PLAIN", "PREC_FP32"])
def test_injected_allocation_failure_leaks_nothing(fdtd, prec):
    import torch

    torch.cuda.init()
    kw = dict(mode=3, size=(96, 96, 96), use_pml=True, pml=8, use_tfsf=True, tfsf_left=14, tfsf_right=14,
              teta=30, phi=45, psi=0, precision=getattr(fdtd, prec))
    eps = np.full((96, 96, 96), 2.0)

    def run():
        with fdtd.Simulation(**kw) as sim:
            sim.set_material("eps", eps)
            sim.step(3)
            sim.sync()
            return sim.field("Ey")

    good = run()   # warms the library's device code and the runtime
    base = _free_bytes()
    failed = 0
    try:
        for after in range(0, 200):
            fdtd.inject_alloc_failure(after)
            try:
                out = run()
            except fdtd.FdtdError as e:
                assert e.status == ERR_NOMEM, (after, e)
                failed += 1
                # whatever the failing call had taken is released again
                assert base - _free_bytes() <= 4 << 20, (after, base - _free_bytes())
                continue
            # enough allocations were allowed: the run completes and is unchanged
            assert np.array_equal(out, good)
            break
        else:
            pytest.fail("the run never completed within 200 allocations")
    finally:
        fdtd.inject_alloc_failure(-1)
    assert failed >= 10   # every allocation up to the last one was made to fail in turn
    assert base - _free_bytes() <= 4 << 20


def test_injected_allocation_failure_in_adjoint_and_batch(fdtd):
    n = 64
    kw = dict(mode=2, size=(n, n), point_source=(20, 32, 0), precision=fdtd.PREC_FP32, **PHYS)
    with fdtd.Simulation(**kw) as sim:
        fdtd.inject_alloc_failure(0)
        try:
            with pytest.raises(fdtd.FdtdError) as e:
                sim.backward(100, 50, (40, 28), (48, 36), fdtd.PREC_FP32)
        finally:
            fdtd.inject_alloc_failure(-1)
        assert e.value.status == ERR_NOMEM, e.value
        j, g = sim.backward(100, 50, (40, 28), (48, 36), fdtd.PREC_FP32)
        assert j > 0 and np.isfinite(g).all()
    fdtd.inject_alloc_failure(3)
    try:
        with pytest.raises(fdtd.FdtdError) as e:
            fdtd.Batch([(40, 40), (50, 30)], **PHYS)
    finally:
        fdtd.inject_alloc_failure(-1)
    assert e.value.status == ERR_NOMEM
