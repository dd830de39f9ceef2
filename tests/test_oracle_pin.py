"""Pins the oracle (oracle/fdtd_oracle.c) before it is trusted as the checker.

1. Against the golden vector the reference's own unit test hard-codes
   (Source/UnitTests/unit-test-internalscheme.cpp, test1D_ExHy): 1-D ExHy,
   200 TF/SF steps; real part = sine source, imaginary part = cosine source.
2. Against fields dumped by the reference CPU double build (committed
   fixtures, tests/golden/make_golden.py).  The dumps carry 15 significant
   digits, so agreement is checked per element at 1e-14 relative.
3. Against the reference binary run live (oracle/_ref/fdtd3d, when built
   here) on the config-1 geometry: 80^3, PML 10, TF/SF 15, 30 steps.
"""
import json
import os

import numpy as np
import pytest

from oracle.oracle import REF_BIN, Oracle, exhy_1d, f32, run_reference

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _per_element_ok(a, r, rel=1e-14):
    return np.all(np.abs(a - r) <= rel * np.abs(r) + 1e-300)


def test_exhy_unit_test_golden_vector():
    g = json.load(open(os.path.join(GOLDEN, "exhy_1d_unit_test.json")))
    s, c = exhy_1d(g["size"], g["tfsf"], g["dx"], g["wavelength"], g["courant"], g["steps"])
    for k, (re, im) in g["ex"].items():
        k = int(k)
        assert abs(s[k] - re) <= 1e-15, (k, s[k], re)
        assert abs(c[k] - im) <= 1e-15, (k, c[k], im)
    # outside the TF/SF box the field is exactly zero
    assert s[6] == 0.0 and s[13] == 0.0


@pytest.mark.parametrize("name", ["ref_dim3_ps", "ref_dim3_pml_tfsf", "ref_dim3_drude", "ref_tmz_pml_tfsf"])
def test_oracle_matches_reference_fixture(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    kw = json.loads(str(z["args"]))
    steps = kw.pop("steps")
    mats = {k[4:]: z[k] for k in z.files if k.startswith("mat_")}
    o = Oracle(materials=mats or None, **kw)
    o.step(steps)
    comps = [k for k in z.files if k in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")]
    assert comps
    for comp in comps:
        a = o.field(comp)
        r = z[comp]
        assert _per_element_ok(a, r), (name, comp, float(np.max(np.abs(a - r))))


@pytest.mark.skipif(not os.path.exists(REF_BIN), reason="reference binary not built (make -C oracle ref)")
def test_oracle_matches_live_reference_config1_geometry():
    kw = dict(mode=3, size=80, use_pml=True, pml=10, use_tfsf=True, tfsf_left=15, tfsf_right=15,
              teta=0, phi=0, psi=0, dx=0.0005, wavelength=0.02, courant=0.5)
    ref, _ = run_reference(steps=30, **kw)
    o = Oracle(**kw)
    o.step(30)
    for comp, r in ref.items():
        assert _per_element_ok(o.field(comp), r), comp


def test_oracle_scalars_are_physical():
    o = Oracle(mode=3, size=12, teta=30, phi=45, psi=0)
    s = o.scalars()
    # float flags are parsed with std::stof, so dx and the Courant factor are float-rounded
    assert s["dt"] == f32(0.0005) * f32(0.5) / 299792458.0
    # oblique propagation is numerically faster than along an axis: pv0 / pv < 1
    assert 0.99 < s["rel_phase_velocity"] < 1.0


def test_unit_test_1d_fixture_is_consistent():
    """unit_test_1d_modes.json (all six 1-D modes, both layouts) holds the same
    ExHy E_CENTERED block as exhy_1d_unit_test.json, and the oracle's 1-D
    ExHy run reproduces it."""
    g = json.load(open(os.path.join(GOLDEN, "unit_test_1d_modes.json")))
    old = json.load(open(os.path.join(GOLDEN, "exhy_1d_unit_test.json")))
    assert sorted(g["modes"]) == ["ExHy", "ExHz", "EyHx", "EyHz", "EzHx", "EzHy"]
    blk = g["modes"]["ExHy"]["E_CENTERED"]
    for k, v in old["ex"].items():
        assert blk[k] == v, k
    s, c = exhy_1d(g["size"], g["tfsf"], g["dx"], g["wavelength"], g["courant"], g["steps"])
    for k, (re, im) in blk.items():
        assert abs(s[int(k)] - re) <= 1e-15 and abs(c[int(k)] - im) <= 1e-15, k


@pytest.mark.skipif(not os.path.exists(REF_BIN), reason="reference binary not built (make -C oracle ref)")
@pytest.mark.parametrize("name", ["ref_dim3_hc_pml_tfsf", "ref_tez_hc_pml_tfsf"])
def test_h_centered_fixtures_match_live_reference(name):
    """The committed H_CENTERED dumps (checked against the CUDA path in the GPU
    tests) are what the reference binary writes for their arguments."""
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    kw = json.loads(str(z["args"]))
    assert kw["layout"] == 1
    mats = {k[4:]: z[k] for k in z.files if k.startswith("mat_")}
    ref, _ = run_reference(materials=mats or None, **kw)
    comps = [k for k in z.files if k in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")]
    assert sorted(comps) == sorted(ref)
    for comp in comps:
        assert np.array_equal(ref[comp], z[comp]), comp
