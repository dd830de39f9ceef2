"""Batched 2-D TMz (one persistent launch per step call, in a CUDA graph)
against the FP64 oracle per instance, and against single-instance runs of
the same configuration through fdtd_step."""
import numpy as np
import pytest

from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

PHYS = dict(use_pml=True, pml=6, dx=0.0005, wavelength=0.02, courant=0.5, teta=90, phi=0, psi=90,
            point_source_mask=1 << 2, point_source_kind=1, point_source_bandwidth=0.5)


def rel_l2(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def instances(seed, count, lo, hi):
    rng = np.random.default_rng(seed)
    sizes = [(int(rng.integers(lo, hi + 1)), int(rng.integers(lo, hi + 1))) for _ in range(count)]
    eps = []
    for nx, ny in sizes:
        blocks = rng.uniform(1, 12, ((nx + 7) // 8, (ny + 7) // 8)).astype(np.float32).astype(np.float64)
        eps.append(np.kron(blocks, np.ones((8, 8)))[:nx, :ny].copy())
    return sizes, eps


@pytest.mark.parametrize("steps,split", [(60, (60,)), (70, (1, 29, 40))])
def test_batch_matches_oracle_per_instance(fdtd, steps, split):
    sizes, eps = instances(7, 6, 20, 70)
    with fdtd.Batch(sizes, **PHYS) as b:
        for i, e in enumerate(eps):
            b.set_eps(i, e)
        for n in split:            # several launches continue one another
            b.step(n)
        b.sync()
        for i, ((nx, ny), e) in enumerate(zip(sizes, eps)):
            o = Oracle(mode=2, size=(nx, ny), point_source=(nx // 2, ny // 2), materials={"eps": e}, **PHYS)
            o.step(steps)
            g = np.concatenate([b.field(i, c).ravel() for c in ("Ez",)])
            r = o.field("Ez").ravel()
            assert rel_l2(g, r) <= 1e-5, (i, rel_l2(g, r))
            gh = np.concatenate([b.field(i, c).ravel() for c in ("Hx", "Hy")])
            rh = np.concatenate([o.field(c).ravel() for c in ("Hx", "Hy")])
            assert rel_l2(gh, rh) <= 1e-5, (i, rel_l2(gh, rh))


def test_batch_equals_single_runs_and_tuner(fdtd):
    sizes, eps = instances(11, 5, 40, 100)
    with fdtd.Batch(sizes, **PHYS) as b:
        for i, e in enumerate(eps):
            b.set_eps(i, e)
        choice = b.tune(4)
        assert len(choice) == 3 and choice[0] in (16, 32, 64, 128)
        b.step(50)
        b.sync()
        info = b.info()
        assert info["cells"] == sum(nx * ny for nx, ny in sizes)
        for i, ((nx, ny), e) in enumerate(zip(sizes, eps)):
            with fdtd.Simulation(mode=2, size=(nx, ny), point_source=(nx // 2, ny // 2), precision=fdtd.PREC_FP32,
                                 materials={"eps": e}, **PHYS) as s:
                s.step(50)
                for c in ("Ez", "Hx", "Hy"):
                    a, r = b.field(i, c), s.field(c)
                    assert rel_l2(a, r) <= 1e-6, (i, c, rel_l2(a, r))


def test_batch_rejects_unsupported(fdtd):
    with pytest.raises(fdtd.FdtdError):
        fdtd.Batch([(30, 30)], use_tfsf=True, tfsf_left=5, tfsf_right=5, **{k: v for k, v in PHYS.items()})
    with pytest.raises(fdtd.FdtdError):
        fdtd.Batch([(30, 30)], precision=fdtd.PREC_FP64_PLAIN, **PHYS)
