"""The TMA-pipelined one-sweep 3-D kernel (sweep3d_tma) against the oracle.

The kernel serves the FP32 and FP16-storage forms of 3-D grids whose z
extent is a multiple of one 16-byte unit (4 FP32 / 8 FP16 cells) when mu is
uniform and there are no metamaterials.  These cases are built so that its
tile seams are exercised: several 128-cell z tiles, partial y tiles, x
chunks of different lengths, point sources on the z ring cell and on both
sides of a tile seam, PML and TF/SF faces crossing tiles, uniform and
per-cell permittivity.  Every test also checks that the kernel actually ran
(fdtd_step_kernel), so a silent fallback cannot pass.

Bars: FP32 <= 1e-5 relative L2 per field family against the FP64 oracle,
FP16 storage <= 2e-2; FP32 sweep vs the register-blocked FP32 kernel
<= 1e-6 (same formulation, different rounding of the TF/SF correction).
"""
import numpy as np
import pytest

from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

COMPS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")

SWEEP_CASES = {
    # three z tiles, partial last y tile, oblique plane wave, sphere of eps 4,
    # point sources on the z ring cell of tile 0 (Ex, Ey) and H on Hz
    "z_tiles_ring_source": dict(
        kw=dict(mode=3, size=(20, 19, 264), use_pml=True, pml=(3, 3, 5), use_tfsf=True, tfsf_left=(5, 5, 7),
                tfsf_right=(6, 5, 8), teta=30, phi=45, psi=20, point_source=(9, 8, 128),
                point_source_mask=(1 << 0) | (1 << 1) | (1 << 5)),
        sphere=((10, 9, 130), 36)),
    # a source on the last cell of a tile and TF/SF faces at the seam
    "seam_source": dict(
        kw=dict(mode=3, size=(17, 24, 136), use_pml=True, pml=4, use_tfsf=True, tfsf_left=(6, 6, 8),
                tfsf_right=(5, 7, 8), teta=60, phi=20, psi=45, point_source=(8, 11, 127),
                point_source_mask=(1 << 2) | (1 << 3) | (1 << 4)),
        sphere=((8, 12, 127), 20)),
    # uniform permittivity (no eps buffer), PML only, source at z = 256
    "uniform_eps_pml": dict(
        kw=dict(mode=3, size=(14, 13, 272), use_pml=True, pml=(3, 4, 6), point_source=(7, 6, 256),
                point_source_mask=1 << 1, teta=0, phi=0, psi=0),
        sphere=None),
    # TF/SF faces right next to the PML: the band overlaps PML cells, so the
    # corrections stay inside the sweep
    "tfsf_touching_pml": dict(
        kw=dict(mode=3, size=(18, 17, 136), use_pml=True, pml=(3, 3, 4), use_tfsf=True, tfsf_left=(4, 4, 5),
                tfsf_right=(4, 4, 5), teta=40, phi=10, psi=30),
        sphere=((9, 8, 60), 25)),
    # TF/SF without PML, axis-aligned incidence, grid smaller than one tile
    "small_tfsf": dict(
        kw=dict(mode=3, size=(16, 15, 40), use_tfsf=True, tfsf_left=(4, 4, 5), tfsf_right=(5, 4, 6),
                teta=0, phi=0, psi=0),
        sphere=((8, 7, 20), 10)),
}


def _materials(case):
    spec = SWEEP_CASES[case]
    if spec["sphere"] is None:
        return None
    (cx, cy, cz), r2 = spec["sphere"]
    x, y, z = np.indices(spec["kw"]["size"])
    return {"eps": np.where((x - cx) ** 2 + (y - cy) ** 2 + (z - cz) ** 2 < r2, 4.0, 1.0)}


def _rel(g, r):
    n = np.linalg.norm(r)
    return np.linalg.norm(g - r) / n if n > 0 else np.linalg.norm(g)


def _run(fdtd, case, prec, steps):
    kw = SWEEP_CASES[case]["kw"]
    with fdtd.Simulation(materials=_materials(case), precision=prec, **kw) as sim:
        sim.step(steps)
        sim.sync()
        kernel = sim.step_kernel
        fields = {c: sim.field(c) for c in COMPS}
    return kernel, fields


_ORACLE_CACHE = {}


def _oracle(case, steps):
    key = (case, steps)
    if key not in _ORACLE_CACHE:
        kw = SWEEP_CASES[case]["kw"]
        o = Oracle(materials=_materials(case), **kw)
        o.step(steps)
        _ORACLE_CACHE[key] = {c: o.field(c) for c in COMPS}
        o.close()
    return _ORACLE_CACHE[key]


def _family_err(got, ref):
    errs = {}
    for fam in ("E", "H"):
        cs = [c for c in COMPS if c[0] == fam]
        g = np.concatenate([got[c].ravel() for c in cs])
        r = np.concatenate([ref[c].ravel() for c in cs])
        assert np.all(np.isfinite(g))
        errs[fam] = _rel(g, r)
    return errs


@pytest.mark.parametrize("case", sorted(SWEEP_CASES))
@pytest.mark.parametrize("prec,tol", [(1, 1e-5), (2, 2e-2)])
def test_sweep_matches_oracle(fdtd, case, prec, tol):
    steps = 36
    kernel, got = _run(fdtd, case, prec, steps)
    assert kernel == "sweep3d_tma", kernel
    errs = _family_err(got, _oracle(case, steps))
    assert errs["E"] <= tol and errs["H"] <= tol, (case, prec, errs)


@pytest.mark.parametrize("chunk", [1, 3, 7, 64])
def test_sweep_x_chunks_agree(fdtd, monkeypatch, chunk):
    """Every x chunk (one plane per item up to the whole grid) gives the
    oracle's fields (FP32)."""
    case = "z_tiles_ring_source"
    monkeypatch.setenv("FDTDB_SWEEP_CHUNK", str(chunk))
    kernel, got = _run(fdtd, case, 1, 30)
    assert kernel == "sweep3d_tma", kernel
    errs = _family_err(got, _oracle(case, 30))
    assert errs["E"] <= 1e-5 and errs["H"] <= 1e-5, (chunk, errs)


@pytest.mark.parametrize("case", ["z_tiles_ring_source", "seam_source"])
def test_sweep_matches_register_blocked_kernel(fdtd, monkeypatch, case):
    steps = 30
    kernel, got = _run(fdtd, case, 1, steps)
    assert kernel == "sweep3d_tma"
    monkeypatch.setenv("FDTDB_SWEEP", "0")
    kernel0, ref = _run(fdtd, case, 1, steps)
    assert kernel0 == "fused3d_regblock", kernel0
    for c in COMPS:
        assert _rel(got[c], ref[c]) <= 1e-6, (case, c, _rel(got[c], ref[c]))


def test_sweep_repeated_launches_reset_work_counter(fdtd):
    """Many one-step calls in a row: each launch must see a fresh work queue
    (the last CTA of a launch resets it), or the fields would stop
    changing."""
    kw = SWEEP_CASES["uniform_eps_pml"]["kw"]
    o = Oracle(**kw)
    with fdtd.Simulation(precision=1, **kw) as sim:
        for _ in range(25):
            sim.step(1)
        sim.sync()
        assert sim.step_kernel == "sweep3d_tma"
        got = {c: sim.field(c) for c in COMPS}
    o.step(25)
    ref = {c: o.field(c) for c in COMPS}
    o.close()
    errs = _family_err(got, ref)
    assert errs["E"] <= 1e-5 and errs["H"] <= 1e-5, errs


@pytest.mark.parametrize("case", ["z_tiles_ring_source", "small_tfsf"])
def test_sweep_inline_tfsf_matches_oracle(fdtd, monkeypatch, case):
    """TF/SF corrections inside the sweep (the path for bands that reach the
    PML) agree with the oracle as the post pass does."""
    monkeypatch.setenv("FDTDB_TFSF_POST", "0")
    kernel, got = _run(fdtd, case, 1, 36)
    assert kernel == "sweep3d_tma", kernel
    errs = _family_err(got, _oracle(case, 36))
    assert errs["E"] <= 1e-5 and errs["H"] <= 1e-5, (case, errs)


def _drude_block_case():
    """A Drude block (eps_inf = 1, omega_p = 2 pi 30 GHz, gamma = 2 pi 1 GHz
    for eps and mu) two cells inside the TF/SF box, next to a sphere of
    eps = 4, under an oblique plane wave: the sweep runs with the Drude
    fix-up."""
    kw = dict(mode=3, size=(24, 22, 40), use_pml=True, pml=3, use_tfsf=True, tfsf_left=6, tfsf_right=6,
              teta=20, phi=30, psi=10, use_metamaterials=True)
    n = kw["size"]
    om = np.zeros(n)
    ga = np.zeros(n)
    om[8:16, 9:15, 17:25] = np.float32(2 * np.pi * 30e9)
    ga[8:16, 9:15, 17:25] = np.float32(2 * np.pi * 1e9)
    x, y, z = np.indices(n)
    eps = np.where((x - 12) ** 2 + (y - 11) ** 2 + (z - 10) ** 2 < 9, 4.0, 1.0)
    return kw, {"eps": eps, "omegape": om, "omegapm": om, "gammae": ga, "gammam": ga}


@pytest.mark.parametrize("prec,tol", [(1, 1e-5), (2, 2e-2)])
def test_sweep_drude_fixup_matches_oracle(fdtd, monkeypatch, prec, tol):
    """Metamaterials through the sweep: the Drude cells and the H cells next
    to them are recomputed after each sweep step.  FP32 / FP16 storage
    against the FP64 oracle, and FP32 against the register-blocked kernel
    (same formulation) to <= 1e-6."""
    kw, mats = _drude_block_case()
    steps = 60
    monkeypatch.setenv("FDTDB_SWEEP_VERBOSE", "1")
    with fdtd.Simulation(materials=mats, precision=prec, **kw) as sim:
        sim.step(steps)
        sim.sync()
        assert sim.step_kernel == "sweep3d_tma", sim.step_kernel
        got = {c: sim.field(c) for c in COMPS}
    o = Oracle(materials=mats, **kw)
    o.step(steps)
    ref = {c: o.field(c) for c in COMPS}
    o.close()
    errs = _family_err(got, ref)
    assert errs["E"] <= tol and errs["H"] <= tol, (prec, errs)
    if prec == 1:
        monkeypatch.setenv("FDTDB_SWEEP", "0")
        with fdtd.Simulation(materials=mats, precision=prec, **kw) as sim:
            sim.step(steps)
            sim.sync()
            assert sim.step_kernel == "fused3d_regblock", sim.step_kernel
            rb = {c: sim.field(c) for c in COMPS}
        errs = _family_err(got, rb)
        assert errs["E"] <= 1e-6 and errs["H"] <= 1e-6, errs


def test_sweep_drude_in_pml_keeps_register_blocked_kernel(fdtd):
    """Drude cells that reach the PML are not fixed up after the sweep: the
    register-blocked kernel serves the run."""
    kw, mats = _drude_block_case()
    om = np.zeros(kw["size"])
    om[:, :, 17:25] = np.float32(2 * np.pi * 30e9)
    mats = dict(mats, omegape=om, omegapm=om)
    with fdtd.Simulation(materials=mats, precision=1, **kw) as sim:
        sim.step(4)
        sim.sync()
        assert sim.step_kernel == "fused3d_regblock", sim.step_kernel
