"""--use-double-material-precision: eps, mu and the PML sigma on a grid of
twice the resolution, each component averaging the 2 x 2 x 2 fine cells
around it (Source/Layout/YeeGridLayout.h:866-1030,
Source/Layout/Approximation.cpp:34-54, Source/Scheme/SchemeHelper.h:596-718).

* fdtd3d-b200 and the reference CPU build write byte-identical TXT dumps:
  3-D with PML and oblique TF/SF over a fine permittivity map, 3-D with fine
  eps and mu maps and a point source, H_CENTERED, 2-D TMz and TEx, 1-D ExHy.
* A fine map that repeats every coarse cell 2 x 2 x 2 times gives, without
  PML, exactly the run of the coarse map (the eight-point tree reduces to the
  two- and four-point averages).
* FP32 agrees with FP64 to 1e-5 relative L2.
"""
import os
import subprocess

import numpy as np
import pytest

from oracle.oracle import REF_BIN, write_material_txt

pytestmark = pytest.mark.gpu
NAMES = ("x", "y", "z")

# name: (mode flag, kept axes, size, extra flags, materials)
CASES = {
    "3d_pml_tfsf": ("--3d", (0, 1, 2), (14, 12, 16),
                    ["--use-tfsf", "--tfsf-size-left", "x:4", "--same-size-tfsf", "--tfsf-size-right", "x:4",
                     "--angle-teta", "30", "--angle-phi", "40", "--angle-psi", "10"], ("eps",)),
    "3d_mu_point_source": ("--3d", (0, 1, 2), (14, 13, 15),
                           ["--point-source", "x:7,y:6,z:8", "--point-source-ez", "--point-source-hx"],
                           ("eps", "mu")),
    "3d_h_centered": ("--3d", (0, 1, 2), (14, 12, 16),
                      ["--use-tfsf", "--tfsf-size-left", "x:4", "--same-size-tfsf", "--tfsf-size-right", "x:4",
                       "--angle-teta", "30", "--angle-phi", "40", "--angle-psi", "10", "--layout-type", "1"],
                      ("eps",)),
    "tmz": ("--2d-tmz", (0, 1), (28, 24, 1),
            ["--use-tfsf", "--tfsf-size-left", "x:6", "--same-size-tfsf", "--tfsf-size-right", "x:6",
             "--angle-teta", "90", "--angle-phi", "30", "--angle-psi", "90"], ("eps", "mu")),
    "tex": ("--2d-tex", (1, 2), (1, 22, 26),
            ["--use-tfsf", "--tfsf-size-left", "x:6", "--same-size-tfsf", "--tfsf-size-right", "x:6",
             "--angle-teta", "30", "--angle-phi", "90", "--angle-psi", "90"], ("eps",)),
    "exhy": ("--1d-exhy", (2,), (1, 1, 50),
             ["--use-tfsf", "--tfsf-size-left", "x:10", "--same-size-tfsf", "--tfsf-size-right", "x:10",
              "--angle-teta", "0", "--angle-phi", "0", "--angle-psi", "90"], ("eps",)),
}


def _fine_map(case, name):
    _, kept, size, _, _ = CASES[case]
    shape = tuple(2 * size[a] for a in kept)
    rng = np.random.default_rng(len(case) + len(name))
    hi = 4.0 if name == "eps" else 2.0
    return np.where(rng.random(shape) < 0.3, hi, 1.0)


@pytest.mark.parametrize("case", sorted(CASES))
def test_cli_double_material_precision_matches_reference_txt(fdtd, tmp_path, case):
    if not os.path.exists(REF_BIN):
        pytest.skip("reference binary not built")
    flag, kept, size, extra, mats = CASES[case]
    sz = ",".join(f"{NAMES[a]}:{size[a]}" for a in kept)
    flags = [flag, "--size", sz, "--use-pml", "--pml-size", "x:3", "--same-size-pml", "--time-steps", "25",
             "--use-double-material-precision"] + extra + [
        "--save-res", "--save-as-txt", "--manual-save-coords",
        "--save-start-coord", ",".join(f"{NAMES[a]}:0" for a in kept), "--save-end-coord", sz]
    for m in mats:
        write_material_txt(str(tmp_path / f"{m}.txt"), _fine_map(case, m))
        flags += [f"--load-{m}-from-file", str(tmp_path / f"{m}.txt")]
    cli = os.path.join(os.path.dirname(fdtd.__file__), "fdtd3d-b200")
    out = {}
    for name, exe, more in (("ref", REF_BIN, ["--use-ca-cb", "--use-ca-cb-pml"]), ("b200", cli, [])):
        d = tmp_path / name
        d.mkdir()
        r = subprocess.run([exe] + flags + more, cwd=d, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
        out[name] = {f.name: f.read_text() for f in d.iterdir()}
    assert sorted(out["ref"]) == sorted(out["b200"]) and out["ref"]
    for fname, text in out["ref"].items():
        mine = out["b200"][fname]
        if mine != text:
            diffs = [(a, b) for a, b in zip(text.splitlines(), mine.splitlines()) if a != b]
            raise AssertionError(f"{fname}: {len(diffs)} lines differ, first: {diffs[:4]}")


@pytest.mark.parametrize("layout", [0, 1])
def test_repeated_fine_map_equals_coarse_run(fdtd, layout):
    n = (18, 16, 20)
    rng = np.random.default_rng(5)
    eps = np.round(rng.uniform(1, 5, n))
    mu = np.round(rng.uniform(1, 2, n))
    up = lambda a: a.repeat(2, 0).repeat(2, 1).repeat(2, 2)  # noqa: E731
    kw = dict(mode=3, size=n, use_tfsf=True, tfsf_left=4, tfsf_right=4, teta=30, phi=40, psi=10, layout=layout,
              point_source=(9, 8, 10), point_source_mask=1 << 1)
    res = {}
    for dmp, mats in ((False, {"eps": eps, "mu": mu}), (True, {"eps": up(eps), "mu": up(mu)})):
        with fdtd.Simulation(precision=fdtd.PREC_FP64_PLAIN, double_material_precision=dmp, materials=mats,
                             **kw) as sim:
            sim.step(30)
            res[dmp] = {c: sim.field(c) for c in fdtd.COMPONENTS}
    for c in fdtd.COMPONENTS:
        assert np.array_equal(res[True][c].view(np.int64), res[False][c].view(np.int64)), c


def test_fp32_double_material_precision_matches_fp64(fdtd):
    n = (24, 20, 26)
    x, y, z = np.indices(tuple(2 * a for a in n))
    eps = np.where((x - 24) ** 2 + (y - 20) ** 2 + (z - 26) ** 2 < 150, 4.0, 1.0)
    kw = dict(mode=3, size=n, use_pml=True, pml=4, use_tfsf=True, tfsf_left=7, tfsf_right=7, teta=30, phi=40,
              psi=10, double_material_precision=True)
    out = {}
    for prec in (fdtd.PREC_FP64_PLAIN, fdtd.PREC_FP32):
        with fdtd.Simulation(precision=prec, materials={"eps": eps}, **kw) as sim:
            sim.step(40)
            out[prec] = {c: sim.field(c) for c in fdtd.COMPONENTS}
            if prec == fdtd.PREC_FP32:
                assert sim.step_kernel == "per_cell", sim.step_kernel
    for fam in ("E", "H"):
        names = [c for c in fdtd.COMPONENTS if c[0] == fam]
        num = sum(np.sum((out[1][c] - out[0][c]) ** 2) for c in names)
        den = sum(np.sum(out[0][c] ** 2) for c in names)
        assert den > 0
        assert np.sqrt(num / den) <= 1e-5, (fam, np.sqrt(num / den))
