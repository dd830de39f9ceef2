"""Adjoint gradient of the 2-D TMz objective through the C ABI
(fdtd_objective / fdtd_backward).

J(eps) = sum over t < steps of sum over a probe box of Ez_t^2, for a
Gaussian-modulated point source left of a design region of random eps and a
probe to its right (the geometry of the adjoint benchmark, scaled down for
the quick cases).  Checks:
  * the adjoint module's forward run is the library's FP32 TMz step (J from
    fdtd_objective against J summed from fdtd_step + downloads);
  * the FP64 adjoint gradient against central differences of the FP64
    objective (h = 1e-4 on eps);
  * the FP32 adjoint gradient against the FP64 adjoint and against the
    finite differences, <= 1e-3 relative (L2 over the checked cells);
  * the checkpoint interval does not change the result (bitwise);
  * a torch.autograd.Function wrapper (test harness only) returns the
    adjoint gradient and passes a directional-derivative check.
The full-size case (512^2, PML 16, 128^2 design, 4000 steps, checkpoint 200,
32 finite-difference cells) is test_adjoint_full_size.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PREC64 = 0
PREC32 = 1


def geometry(n, pml, design, probe, gap):
    c = n // 2
    d0, d1 = c - design // 2, c - design // 2 + design
    src = (d0 - gap, c)
    p0 = (d1 + gap, c - probe // 2)
    return dict(box=(d0, d1), src=src, probe_lo=p0, probe_hi=(p0[0] + probe, p0[1] + probe))


def config(n, pml, geo, precision):
    return dict(mode=2, size=(n, n), use_pml=True, pml=pml, teta=90, phi=0, psi=90,
                point_source=(geo["src"][0], geo["src"][1], 0), point_source_mask=1 << 2,
                point_source_kind=1, point_source_bandwidth=0.5, precision=precision)


def design_eps(n, geo, seed):
    rng = np.random.default_rng(seed)
    eps = np.ones((n, n))
    d0, d1 = geo["box"]
    eps[d0:d1, d0:d1] = rng.uniform(1.0, 12.0, (d1 - d0, d1 - d0)).astype(np.float32)
    return eps


SMALL = dict(n=96, pml=8, design=24, probe=6, gap=20, steps=400, every=40, seed=5)


def small_setup():
    s = SMALL
    geo = geometry(s["n"], s["pml"], s["design"], s["probe"], s["gap"])
    return s, geo, design_eps(s["n"], geo, s["seed"])


def objective(fdtd, n, pml, geo, eps, steps, precision):
    with fdtd.Simulation(materials={"eps": eps}, **config(n, pml, geo, precision)) as sim:
        return sim.objective(steps, geo["probe_lo"], geo["probe_hi"], precision)


def backward(fdtd, n, pml, geo, eps, steps, every, precision, ctx_precision=PREC32):
    with fdtd.Simulation(materials={"eps": eps}, **config(n, pml, geo, ctx_precision)) as sim:
        return sim.backward(steps, every, geo["probe_lo"], geo["probe_hi"], precision)


def test_adjoint_forward_is_the_library_step(fdtd):
    s, geo, eps = small_setup()
    (px0, py0), (px1, py1) = geo["probe_lo"], geo["probe_hi"]
    with fdtd.Simulation(materials={"eps": eps}, **config(s["n"], s["pml"], geo, PREC32)) as sim:
        j_lib = 0.0
        for _ in range(s["steps"]):
            sim.step(1)
            ez = sim.field("Ez")
            j_lib += float(np.sum(ez[px0:px1, py0:py1] ** 2))
        j_adj = sim.objective(s["steps"], geo["probe_lo"], geo["probe_hi"], PREC32)
    assert j_lib > 0
    assert abs(j_adj - j_lib) <= 1e-6 * j_lib, (j_adj, j_lib)
    j64 = objective(fdtd, s["n"], s["pml"], geo, eps, s["steps"], PREC64)
    assert abs(j64 - j_lib) <= 1e-4 * j_lib, (j64, j_lib)


def test_adjoint_fp64_matches_central_differences(fdtd):
    s, geo, eps = small_setup()
    j, g = backward(fdtd, s["n"], s["pml"], geo, eps, s["steps"], s["every"], PREC64)
    d0, d1 = geo["box"]
    rng = np.random.default_rng(11)
    cells = [(int(a), int(b)) for a, b in rng.integers(d0, d1, (8, 2))]
    h = 1e-4
    for (x, y) in cells:
        ep = eps.copy()
        ep[x, y] += h
        em = eps.copy()
        em[x, y] -= h
        fd = (objective(fdtd, s["n"], s["pml"], geo, ep, s["steps"], PREC64)
              - objective(fdtd, s["n"], s["pml"], geo, em, s["steps"], PREC64)) / (2 * h)
        assert abs(fd - g[x, y]) <= 1e-6 * np.max(np.abs(g)) + 1e-6 * abs(fd), ((x, y), fd, g[x, y])


def test_adjoint_fp32_matches_fp64_adjoint(fdtd):
    s, geo, eps = small_setup()
    j64, g64 = backward(fdtd, s["n"], s["pml"], geo, eps, s["steps"], s["every"], PREC64)
    j32, g32 = backward(fdtd, s["n"], s["pml"], geo, eps, s["steps"], s["every"], PREC32)
    assert abs(j32 - j64) <= 1e-4 * j64
    d0, d1 = geo["box"]
    a, b = g32[d0:d1, d0:d1], g64[d0:d1, d0:d1]
    assert np.linalg.norm(a - b) <= 1e-3 * np.linalg.norm(b), np.linalg.norm(a - b) / np.linalg.norm(b)
    # the whole grid, PML included
    assert np.linalg.norm(g32 - g64) <= 1e-3 * np.linalg.norm(g64)


def test_adjoint_checkpoint_interval_does_not_change_the_result(fdtd):
    s, geo, eps = small_setup()
    ref = None
    for every in (1, 13, s["steps"]):
        j, g = backward(fdtd, s["n"], s["pml"], geo, eps, s["steps"], every, PREC64)
        if ref is None:
            ref = (j, g)
        else:
            assert j == ref[0]
            assert np.array_equal(g, ref[1]), every


def test_adjoint_through_torch_autograd(fdtd):
    """The test-harness wrapper: forward returns J, backward the adjoint gradient."""
    import torch

    s, geo, eps0 = small_setup()

    class Objective(torch.autograd.Function):
        @staticmethod
        def forward(ctx, eps):
            j, g = backward(fdtd, s["n"], s["pml"], geo, eps.detach().cpu().numpy(), s["steps"], s["every"],
                            PREC64)
            ctx.save_for_backward(torch.from_numpy(g))
            return torch.tensor(j, dtype=torch.float64)

        @staticmethod
        def backward(ctx, gout):
            (g,) = ctx.saved_tensors
            return gout * g

    eps = torch.tensor(eps0, dtype=torch.float64, requires_grad=True)
    j = Objective.apply(eps)
    j.backward()
    g = eps.grad.numpy()
    # directional derivative along a random perturbation of the design region
    d0, d1 = geo["box"]
    v = np.zeros_like(eps0)
    v[d0:d1, d0:d1] = np.random.default_rng(3).standard_normal((d1 - d0, d1 - d0))
    h = 1e-5
    jp = objective(fdtd, s["n"], s["pml"], geo, eps0 + h * v, s["steps"], PREC64)
    jm = objective(fdtd, s["n"], s["pml"], geo, eps0 - h * v, s["steps"], PREC64)
    dd = (jp - jm) / (2 * h)
    assert abs(dd - float(np.sum(g * v))) <= 1e-6 * abs(dd), (dd, float(np.sum(g * v)))


def test_adjoint_rejects_unsupported(fdtd):
    with fdtd.Simulation(mode=3, size=12, precision=PREC32) as sim:
        with pytest.raises(fdtd.FdtdError):
            sim.objective(10, (2, 2), (4, 4), PREC32)


def test_adjoint_full_size(fdtd):
    """512^2, PML 16, 128^2 design of eps ~ U[1, 12] at the centre, Gaussian
    source 64 cells left of it, 16^2 probe 64 cells right of it, 4000 steps,
    checkpoint every 200: the FP32 adjoint against central differences
    (h = 1e-4) of the FP64 objective on 32 seeded design cells and against
    the FP64 adjoint, <= 1e-3 relative."""
    n, pml, steps, every = 512, 16, 4000, 200
    geo = geometry(n, pml, 128, 16, 64)
    eps = design_eps(n, geo, 2024)
    j32, g32 = backward(fdtd, n, pml, geo, eps, steps, every, PREC32)
    j64, g64 = backward(fdtd, n, pml, geo, eps, steps, every, PREC64)
    assert j64 > 0 and abs(j32 - j64) <= 1e-4 * j64
    d0, d1 = geo["box"]
    a, b = g32[d0:d1, d0:d1], g64[d0:d1, d0:d1]
    assert np.linalg.norm(a - b) <= 1e-3 * np.linalg.norm(b)
    rng = np.random.default_rng(32)
    cells = [(int(p), int(q)) for p, q in rng.integers(d0, d1, (32, 2))]
    h = 1e-4
    fd = []
    for (x, y) in cells:
        ep = eps.copy()
        ep[x, y] += h
        em = eps.copy()
        em[x, y] -= h
        fd.append((objective(fdtd, n, pml, geo, ep, steps, PREC64)
                   - objective(fdtd, n, pml, geo, em, steps, PREC64)) / (2 * h))
    fd = np.array(fd)
    ga = np.array([g32[c] for c in cells])
    gb = np.array([g64[c] for c in cells])
    assert np.linalg.norm(ga - fd) <= 1e-3 * np.linalg.norm(fd), np.linalg.norm(ga - fd) / np.linalg.norm(fd)
    assert np.linalg.norm(gb - fd) <= 1e-5 * np.linalg.norm(fd), np.linalg.norm(gb - fd) / np.linalg.norm(fd)
