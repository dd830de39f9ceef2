"""The two-step (temporally blocked) sweep (sweep2_tma) against single steps.

The two-step kernel advances pairs of time steps in one pass over HBM.  Its
arithmetic per half-step is the single-step sweep's, and in FP32 the
intermediate step is held in FP32 registers exactly as the single step
stores it, so FP32 pairs must equal two single steps bit for bit.  In FP16
storage the intermediate step stays in FP32 instead of being rounded to
FP16, so the two differ by FP16 rounding (both are checked against FP64).

Grids are chosen to exercise the kernel's tiling: several z tiles (60 own
cells per tile in FP32, 56 in FP16), partial last z and y tiles, several x
chunks, odd step counts (the last step of an odd count is a single step),
random initial fields and per-cell permittivity, and uniform permittivity.
Every test checks that the kernel actually ran (fdtd_step_kernel).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

COMPS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")


def _run(fdtd, monkeypatch, kw, steps, fields, eps, tb2, chunk=None):
    monkeypatch.setenv("FDTDB_TB2", "1" if tb2 else "0")
    # the two-step kernel's x chunk (default 128 planes): short chunks put
    # chunk seams into these small grids
    if chunk:
        monkeypatch.setenv("FDTDB_TB2_CHUNK", str(chunk))
    else:
        monkeypatch.delenv("FDTDB_TB2_CHUNK", raising=False)
    mats = {"eps": eps} if eps is not None else None
    with fdtd.Simulation(materials=mats, **kw) as sim:
        for c, a in fields.items():
            sim.set_field(c, a)
        sim.step(steps)
        sim.sync()
        kernel = sim.step_kernel
        out = {c: sim.field(c).copy() for c in COMPS}
    return out, kernel


def _inputs(shape, seed, with_eps=True):
    rng = np.random.default_rng(seed)
    fields = {c: rng.standard_normal(shape).astype(np.float32).astype(np.float64) for c in COMPS}
    eps = None
    if with_eps:
        blocks = rng.uniform(1.0, 6.0, tuple((s + 5) // 6 for s in shape)).astype(np.float32)
        eps = np.kron(blocks, np.ones((6, 6, 6)))[: shape[0], : shape[1], : shape[2]].astype(np.float64)
    return fields, eps


CASES = {
    # 3 z tiles (the last partial), 5 y tiles (the last partial), 3 x chunks
    "tiles": dict(size=(70, 58, 132), steps=9, eps=True, chunk=32),
    # an odd number of updates (the last a single step), uniform permittivity,
    # one partial z tile
    "odd_uniform": dict(size=(23, 19, 40), steps=8, eps=False),
    # nz just past one tile's own cells and a long x extent (two chunks of
    # the default length)
    "long_x": dict(size=(150, 16, 64), steps=7, eps=True),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_fp32_pairs_equal_single_steps(fdtd, monkeypatch, case):
    spec = CASES[case]
    shape = spec["size"]
    fields, eps = _inputs(shape, 3 + len(case), spec["eps"])
    kw = dict(mode=3, size=shape, precision=fdtd.PREC_FP32)
    got, k2 = _run(fdtd, monkeypatch, kw, spec["steps"], fields, eps, True, spec.get("chunk"))
    ref, k1 = _run(fdtd, monkeypatch, kw, spec["steps"], fields, eps, False)
    assert k1 == "sweep3d_tma"
    # steps from t = 0 update the fields steps - 1 times (none at t = 0); an
    # odd number of updates ends with one single step
    assert k2 == ("sweep3d_tma" if (spec["steps"] - 1) % 2 else "sweep2_tma")
    for c in COMPS:
        assert np.array_equal(got[c], ref[c]), (case, c, float(np.max(np.abs(got[c] - ref[c]))))


def test_two_step_kernel_runs_for_even_counts(fdtd, monkeypatch):
    shape = (30, 20, 72)
    fields, eps = _inputs(shape, 41)
    kw = dict(mode=3, size=shape, precision=fdtd.PREC_FP32)
    _, kernel = _run(fdtd, monkeypatch, kw, 5, fields, eps, True)
    assert kernel == "sweep2_tma"


FP16_CASES = {   # nz a multiple of 8 (one 16-byte unit of halves)
    "tiles": dict(size=(70, 58, 136), steps=9, eps=True),
    "long_x": dict(size=(150, 16, 64), steps=7, eps=True),
}


@pytest.mark.parametrize("case", sorted(FP16_CASES))
def test_fp16_storage_pairs_against_fp32(fdtd, monkeypatch, case):
    spec = FP16_CASES[case]
    shape = spec["size"]
    fields, eps = _inputs(shape, 5 + len(case), spec["eps"])
    # values representable in FP16 storage (H is stored as eta0 * H)
    fields = {c: (a * 0.1).astype(np.float16).astype(np.float64) if c[0] == "E" else
              ((a * 0.1 * 376.730313461770655).astype(np.float16).astype(np.float64) / 376.730313461770655)
              for c, a in fields.items()}
    kw16 = dict(mode=3, size=shape, precision=fdtd.PREC_FP16S)
    kw32 = dict(mode=3, size=shape, precision=fdtd.PREC_FP32)
    got, k2 = _run(fdtd, monkeypatch, kw16, spec["steps"], fields, eps, True)
    one, _ = _run(fdtd, monkeypatch, kw16, spec["steps"], fields, eps, False)
    ref, _ = _run(fdtd, monkeypatch, kw32, spec["steps"], fields, eps, False)
    assert k2 == "sweep2_tma"
    for fam in (COMPS[:3], COMPS[3:]):
        r = np.concatenate([ref[c].ravel() for c in fam])
        g2 = np.concatenate([got[c].ravel() for c in fam])
        g1 = np.concatenate([one[c].ravel() for c in fam])
        for g in (g2, g1):
            assert np.linalg.norm(g - r) / np.linalg.norm(r) <= 2e-2
        # keeping the middle step in FP32 is no less accurate than rounding it to FP16
        assert np.linalg.norm(g2 - r) <= 1.05 * np.linalg.norm(g1 - r)


PML_CASES = {
    # PML on every face (x / y PML items and z PML columns), two partial tiles
    "pml_all_faces": dict(size=(62, 44, 128), pml=(5, 6, 7), steps=9),
    # thick z PML only in the last z tile, thin x / y PML, odd update count
    "pml_thick_z": dict(size=(40, 30, 120), pml=(3, 3, 16), steps=8),
    # a core of several two-step tiles and x chunks inside a PML shell of
    # several single-step tiles on every side
    "pml_large_core": dict(size=(150, 96, 200), pml=(10, 9, 12), steps=9, chunk=40),
}


@pytest.mark.parametrize("case", sorted(PML_CASES))
def test_fp32_pairs_with_pml_match_single_steps(fdtd, monkeypatch, case):
    """With PML, the x / y PML slabs (and a 2-cell margin) take two single
    steps through a third buffer set while the two-step kernel advances the
    rest; it evaluates the z PML cells with the general PML form, where the
    single-step kernel uses a rearranged form on cells whose only PML axis is
    z: the two agree to FP32 rounding (<= 1e-6 relative L2 per field family)
    and the auxiliary state they carry agrees as well (checked through the
    fields of later steps)."""
    spec = PML_CASES[case]
    shape = spec["size"]
    fields, eps = _inputs(shape, 17 + len(case))
    kw = dict(mode=3, size=shape, use_pml=True, pml=spec["pml"], precision=fdtd.PREC_FP32)
    got, k2 = _run(fdtd, monkeypatch, kw, spec["steps"], fields, eps, True, spec.get("chunk"))
    ref, k1 = _run(fdtd, monkeypatch, kw, spec["steps"], fields, eps, False)
    assert k1 == "sweep3d_tma"
    assert k2 == ("sweep3d_tma" if (spec["steps"] - 1) % 2 else "sweep2_tma")
    for fam in (COMPS[:3], COMPS[3:]):
        r = np.concatenate([ref[c].ravel() for c in fam])
        g = np.concatenate([got[c].ravel() for c in fam])
        err = np.linalg.norm(g - r) / np.linalg.norm(r)
        assert err <= 1e-6, (case, fam, err)
    # long enough for waves to cross the PML and come back
    got, _ = _run(fdtd, monkeypatch, kw, 61, fields, eps, True)
    ref, _ = _run(fdtd, monkeypatch, kw, 61, fields, eps, False)
    for fam in (COMPS[:3], COMPS[3:]):
        r = np.concatenate([ref[c].ravel() for c in fam])
        g = np.concatenate([got[c].ravel() for c in fam])
        assert np.linalg.norm(g - r) / np.linalg.norm(r) <= 1e-5, (case, fam)


def _sphere(shape, frac=0.3):
    c = [np.arange(n) + 0.5 - n / 2.0 for n in shape]
    r2 = (frac * min(shape)) ** 2
    return np.where(c[0][:, None, None] ** 2 + c[1][None, :, None] ** 2 + c[2][None, None, :] ** 2 < r2, 4.0, 1.0)


TFSF_CASES = {
    # PML shell and core, oblique plane wave, dielectric sphere
    "pml_tfsf_sphere": dict(kw=dict(size=(96, 90, 120), use_pml=True, pml=6, use_tfsf=True, tfsf_left=22,
                                    tfsf_right=22, teta=30, phi=45, psi=0), steps=61),
    # no PML (the whole grid two-step), another polarisation
    "tfsf_no_pml": dict(kw=dict(size=(40, 36, 64), use_tfsf=True, tfsf_left=(8, 7, 9), tfsf_right=(7, 8, 9),
                                teta=60, phi=20, psi=45), steps=41),
}


@pytest.mark.parametrize("case", sorted(TFSF_CASES))
def test_fp32_pairs_with_tfsf(fdtd, monkeypatch, case):
    """The pair's TF/SF corrections are added after the uncorrected pair as
    its linear response (four passes over the TF/SF band): the result agrees
    with single steps whose corrections are added after each step to FP32
    rounding (<= 1e-6 per field family) and with the FP64 oracle to the
    FP32 bar (1e-5)."""
    from oracle.oracle import Oracle

    spec = TFSF_CASES[case]
    kw = dict(mode=3, dx=0.0005, wavelength=0.02, courant=0.5, **spec["kw"])
    shape = kw["size"]
    eps = _sphere(shape)
    got, k2 = _run(fdtd, monkeypatch, dict(kw, precision=fdtd.PREC_FP32), spec["steps"], {}, eps, True)
    ref, k1 = _run(fdtd, monkeypatch, dict(kw, precision=fdtd.PREC_FP32), spec["steps"], {}, eps, False)
    assert k1 == "sweep3d_tma"
    assert k2 == "sweep2_tma"
    o = Oracle(materials={"eps": eps}, **kw)
    o.step(spec["steps"])
    for fam in (COMPS[:3], COMPS[3:]):
        r = np.concatenate([ref[c].ravel() for c in fam])
        g = np.concatenate([got[c].ravel() for c in fam])
        assert np.linalg.norm(r) > 0
        assert np.linalg.norm(g - r) / np.linalg.norm(r) <= 1e-6, (case, fam)
        ro = np.concatenate([o.field(c).ravel() for c in fam])
        assert np.linalg.norm(g - ro) / np.linalg.norm(ro) <= 1e-5, (case, fam)


def test_fp16_storage_pairs_with_pml_and_tfsf(fdtd, monkeypatch):
    """FP16 storage through the whole two-step scheme (PML shell, core, TF/SF
    pair corrections) against the FP32 single-step form: within the FP16
    bar (2e-2 per family), and no farther than FP16 single steps are."""
    kw = dict(mode=3, size=(96, 90, 120), use_pml=True, pml=6, use_tfsf=True, tfsf_left=22, tfsf_right=22,
              teta=30, phi=45, psi=0, dx=0.0005, wavelength=0.02, courant=0.5)
    eps = _sphere(kw["size"])
    got, k2 = _run(fdtd, monkeypatch, dict(kw, precision=fdtd.PREC_FP16S), 61, {}, eps, True)
    one, _ = _run(fdtd, monkeypatch, dict(kw, precision=fdtd.PREC_FP16S), 61, {}, eps, False)
    ref, _ = _run(fdtd, monkeypatch, dict(kw, precision=fdtd.PREC_FP32), 61, {}, eps, False)
    assert k2 == "sweep2_tma"
    for fam in (COMPS[:3], COMPS[3:]):
        r = np.concatenate([ref[c].ravel() for c in fam])
        g2 = np.concatenate([got[c].ravel() for c in fam])
        g1 = np.concatenate([one[c].ravel() for c in fam])
        assert np.linalg.norm(g2 - r) / np.linalg.norm(r) <= 2e-2
        assert np.linalg.norm(g2 - r) <= 1.05 * np.linalg.norm(g1 - r)



def test_tfsf_box_near_the_pml_keeps_single_steps_correct(fdtd, monkeypatch):
    """A TF/SF box two cells from the PML: the pair's corrections would reach
    the single-step shell, so the plan keeps single steps (the two-step path
    declines the grid) and the fields equal the single-step path's."""
    kw = dict(mode=3, size=(48, 44, 64), use_pml=True, pml=6, use_tfsf=True, tfsf_left=8, tfsf_right=8,
              teta=30, phi=45, psi=0, dx=0.0005, wavelength=0.02, courant=0.5, precision=fdtd.PREC_FP32)
    eps = _sphere(kw["size"])
    got, k2 = _run(fdtd, monkeypatch, kw, 30, {}, eps, True)
    ref, k1 = _run(fdtd, monkeypatch, kw, 30, {}, eps, False)
    assert k1 == "sweep3d_tma"
    if k2 == "sweep2_tma":
        for fam in (COMPS[:3], COMPS[3:]):
            r = np.concatenate([ref[c].ravel() for c in fam])
            g = np.concatenate([got[c].ravel() for c in fam])
            assert np.linalg.norm(g - r) / np.linalg.norm(r) <= 1e-6
    else:
        for c in COMPS:
            np.testing.assert_array_equal(got[c], ref[c])


@pytest.mark.parametrize("splits", [(7, 8, 9), (2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2), (24,)])
def test_any_split_of_the_steps_agrees(fdtd, monkeypatch, splits):
    """fdtd_step calls of any lengths (pairs inside each call, a single step
    for an odd remainder) against one single-step run of the same total:
    PML, TF/SF and a sphere, per field family <= 1e-6."""
    kw = dict(mode=3, size=(96, 90, 120), use_pml=True, pml=6, use_tfsf=True, tfsf_left=22, tfsf_right=22,
              teta=30, phi=45, psi=0, dx=0.0005, wavelength=0.02, courant=0.5, precision=fdtd.PREC_FP32)
    eps = _sphere(kw["size"])
    total = sum(splits)
    ref, _ = _run(fdtd, monkeypatch, kw, total, {}, eps, False)
    monkeypatch.setenv("FDTDB_TB2", "1")
    with fdtd.Simulation(materials={"eps": eps}, **kw) as sim:
        kernels = set()
        for n in splits:
            sim.step(n)
            kernels.add(sim.step_kernel)
        sim.sync()
        got = {c: sim.field(c).copy() for c in COMPS}
    # a call whose last update is the second of a pair reports the pair kernel
    assert "sweep2_tma" in kernels or splits == (24,), kernels
    for fam in (COMPS[:3], COMPS[3:]):
        r = np.concatenate([ref[c].ravel() for c in fam])
        g = np.concatenate([got[c].ravel() for c in fam])
        assert np.linalg.norm(g - r) / np.linalg.norm(r) <= 1e-6, (splits, fam)
