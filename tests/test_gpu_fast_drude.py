"""Drude media (metamaterials) in the FP32 / FP16-storage per-cell kernels.

The per-cell kernels serve what the one-sweep 3-D kernels do not: the 2-D
and 1-D modes, the H_CENTERED layout, non-uniform mu.  A Drude cell (a
nonzero plasma frequency or collision rate on the component's averaging
stencil, getMetaMaterial) takes the reference's metamaterial PML path
(InternalScheme.inc.h:2452-2640): the curl step of X, the Drude recurrence to
Z with b0 .. a2 (:2527-2532) and F from Z with modifier 1.  Each case runs a
Drude block under a TF/SF plane wave with PML against the FP64 plain form
(bit-identical to the reference build): relative L2 per field family
<= 1e-5 (FP32) and <= 2e-2 (FP16 storage), and the block must matter (the
fields differ from a run without it).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

OM = np.float32(2 * np.pi * 30e9)
GA = np.float32(2 * np.pi * 1e9)


def _case(name):
    if name == "tmz":
        kw = dict(mode=2, size=(48, 44), use_pml=True, pml=5, use_tfsf=True, tfsf_left=9, tfsf_right=9,
                  teta=90, phi=30, psi=90)
        shape = (48, 44)
        blk = (slice(18, 30), slice(16, 28))
        comps = ("Ez", "Hx", "Hy")
    elif name == "tez":
        kw = dict(mode=6, size=(46, 40), use_pml=True, pml=5, use_tfsf=True, tfsf_left=9, tfsf_right=9,
                  teta=90, phi=35, psi=0)
        shape = (46, 40)
        blk = (slice(17, 29), slice(14, 26))
        comps = ("Ex", "Ey", "Hz")
    elif name == "eyhz":
        kw = dict(mode=13, size=(120, 1, 1), use_pml=True, pml=8, use_tfsf=True, tfsf_left=14, tfsf_right=14,
                  teta=90, phi=0, psi=0)
        shape = (120,)
        blk = (slice(50, 70),)
        comps = ("Ey", "Hz")
    elif name == "dim3_h_centered":
        kw = dict(mode=3, size=(22, 20, 24), use_pml=True, pml=3, use_tfsf=True, tfsf_left=6, tfsf_right=6,
                  teta=20, phi=30, psi=10, layout=1)
        shape = (22, 20, 24)
        blk = (slice(8, 14), slice(8, 13), slice(9, 15))
        comps = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
    else:   # dim3 with a permeability map: the per-cell kernels
        kw = dict(mode=3, size=(22, 20, 24), use_pml=True, pml=3, use_tfsf=True, tfsf_left=6, tfsf_right=6,
                  teta=20, phi=30, psi=10)
        shape = (22, 20, 24)
        blk = (slice(8, 14), slice(8, 13), slice(9, 15))
        comps = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
    om = np.zeros(shape)
    ga = np.zeros(shape)
    om[blk] = OM
    ga[blk] = GA
    mats = {"omegape": om, "omegapm": om, "gammae": ga, "gammam": ga}
    if name == "dim3_mu":
        mu = np.ones(shape)
        mu[4:10, 4:9, 4:10] = 2.0
        mats["mu"] = mu
    return dict(kw, use_metamaterials=True), mats, comps


def _run(fdtd, kw, mats, prec, steps, comps):
    with fdtd.Simulation(materials=mats, precision=prec, **kw) as sim:
        sim.step(steps)
        sim.sync()
        kernel = sim.step_kernel
        out = {c: sim.field(c).copy() for c in comps}
    return out, kernel


def _fam(a, b, names):
    r = np.concatenate([b[c].ravel() for c in names])
    g = np.concatenate([a[c].ravel() for c in names])
    return np.linalg.norm(g - r) / np.linalg.norm(r)


@pytest.mark.parametrize("name", ["tmz", "tez", "eyhz", "dim3_h_centered", "dim3_mu"])
def test_fp32_per_cell_drude_matches_fp64(fdtd, name):
    kw, mats, comps = _case(name)
    steps = 120 if kw["mode"] != 3 else 50
    ref, k64 = _run(fdtd, kw, mats, fdtd.PREC_FP64_PLAIN, steps, comps)
    got, k32 = _run(fdtd, kw, mats, fdtd.PREC_FP32, steps, comps)
    assert k64 == "plain_fp64" and k32 == "per_cell", (k64, k32)
    fams = [tuple(c for c in comps if c[0] == f) for f in "EH"]
    for fam in fams:
        assert _fam(got, ref, fam) <= 1e-5, (name, fam, _fam(got, ref, fam))
    # the Drude block changes the fields
    plain = {k: v for k, v in mats.items() if k in ("eps", "mu")}
    kw0 = dict(kw, use_metamaterials=False)
    free, _ = _run(fdtd, kw0, plain or None, fdtd.PREC_FP64_PLAIN, steps, comps)
    assert max(_fam(free, ref, fam) for fam in fams) > 1e-3


def test_fp16_storage_per_cell_drude(fdtd):
    kw, mats, comps = _case("tmz")
    ref, _ = _run(fdtd, kw, mats, fdtd.PREC_FP64_PLAIN, 120, comps)
    got, k = _run(fdtd, kw, mats, fdtd.PREC_FP16S, 120, comps)
    assert k == "per_cell"
    for fam in (("Ez",), ("Hx", "Hy")):
        assert _fam(got, ref, fam) <= 2e-2, (fam, _fam(got, ref, fam))
