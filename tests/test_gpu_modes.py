"""The six 2-D modes (Dim2_TEx .. Dim2_TMz) and the six 1-D modes
(Dim1_ExHy .. Dim1_EzHy) against the reference CPU build
(oracle/_ref/fdtd3d, all modes compiled in).

* fdtd3d-b200 (the FP64 plain form) and the reference write byte-identical
  TXT dumps (15 significant digits) for the same flags: PML, TF/SF plane
  wave at an oblique in-plane angle, a permittivity map from a TXT file,
  and, in a second set, a point source on every component of the mode.
* The FP32 form through the C ABI agrees with the reference to <= 1e-5
  relative L2 per field family.
The angles follow each mode's own plane or axis (TEx/TMx: phi = 90,
TEy/TMy: phi = 0, TEz/TMz: teta = 90; the 1-D modes' fixed directions;
Source/Layout/YeeGridLayout.cpp:2050-2580).
"""
import os
import subprocess

import numpy as np
import pytest

from oracle.oracle import REF_BIN, mode_axes, run_reference, write_material_txt

pytestmark = pytest.mark.gpu

MODES = {  # mode: (flag, components, teta, phi, psi)
    4: ("--2d-tex", ("Ey", "Ez", "Hx"), 30, 90, 90),
    5: ("--2d-tey", ("Ex", "Ez", "Hy"), 25, 0, 90),
    6: ("--2d-tez", ("Ex", "Ey", "Hz"), 90, 35, 0),
    7: ("--2d-tmx", ("Ex", "Hy", "Hz"), 40, 90, 0),
    8: ("--2d-tmy", ("Ey", "Hx", "Hz"), 20, 0, 0),
    2: ("--2d-tmz", ("Ez", "Hx", "Hy"), 90, 30, 90),
    10: ("--1d-exhy", ("Ex", "Hy"), 0, 0, 90),
    11: ("--1d-exhz", ("Ex", "Hz"), 90, 90, 0),
    12: ("--1d-eyhx", ("Ey", "Hx"), 0, 90, 90),
    13: ("--1d-eyhz", ("Ey", "Hz"), 90, 0, 0),
    14: ("--1d-ezhx", ("Ez", "Hx"), 90, 90, 90),
    15: ("--1d-ezhy", ("Ez", "Hy"), 90, 0, 90),
}
SIZE = (22, 19, 24)      # x, y, z; a 2-D mode drops one axis, a 1-D mode two
NAMES = ("x", "y", "z")


def _need_ref():
    if not os.path.exists(REF_BIN):
        pytest.skip("reference binary not built")


def _plane_shape(mode):
    return tuple(SIZE[a] for a in mode_axes(mode))


def _eps_map(mode, seed):
    rng = np.random.default_rng(seed)
    return np.where(rng.random(_plane_shape(mode)) < 0.35, 4.0, 1.0)


def _flags(mode, steps, source):
    flag, comps, teta, phi, psi = MODES[mode]
    size = ",".join(f"{n}:{v}" for n, v in zip(NAMES, SIZE))
    f = [flag, "--size", size, "--use-pml", "--pml-size", "x:3", "--same-size-pml",
         "--use-tfsf", "--tfsf-size-left", "x:5", "--same-size-tfsf", "--tfsf-size-right", "x:6",
         "--angle-teta", str(teta), "--angle-phi", str(phi), "--angle-psi", str(psi),
         "--dx", "0.0005", "--wavelength", "0.02", "--courant-factor", "0.5", "--time-steps", str(steps),
         "--save-res", "--save-as-txt", "--manual-save-coords",
         "--save-start-coord", "x:0,y:0,z:0", "--save-end-coord", size]
    if source:
        ps = [9, 8, 11]
        f += ["--point-source", ",".join(f"{n}:{v}" for n, v in zip(NAMES, ps))]
        f += [f"--point-source-{c.lower()}" for c in comps]
    return f


@pytest.mark.parametrize("source", [False, True], ids=["tfsf", "point_source"])
@pytest.mark.parametrize("mode", sorted(MODES), ids=[MODES[m][0][2:] for m in sorted(MODES)])
def test_cli_mode_matches_reference_txt(fdtd, tmp_path, mode, source):
    _need_ref()
    cli = os.path.join(os.path.dirname(fdtd.__file__), "fdtd3d-b200")
    eps_file = tmp_path / "eps.txt"
    write_material_txt(str(eps_file), _eps_map(mode, mode))
    flags = _flags(mode, 30, source) + ["--load-eps-from-file", str(eps_file)]
    out = {}
    for name, exe, extra in (("ref", REF_BIN, ["--use-ca-cb", "--use-ca-cb-pml"]), ("b200", cli, [])):
        d = tmp_path / name
        d.mkdir()
        r = subprocess.run([exe] + flags + extra, cwd=d, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
        out[name] = {f.name: f.read_text() for f in d.iterdir()}
    names = sorted(out["ref"])
    assert names == sorted(out["b200"])
    assert len(names) == len(MODES[mode][1]), names
    for fname in names:
        ref, mine = out["ref"][fname], out["b200"][fname]
        assert ref.count("\n") == np.prod(_plane_shape(mode))
        if mine != ref:
            diffs = [(a, b) for a, b in zip(ref.splitlines(), mine.splitlines()) if a != b]
            raise AssertionError(f"{fname}: {len(diffs)} lines differ, first: {diffs[:4]}")
        # the run must carry signal in every component of the mode
        vals = np.array([float(line.split()[-1]) for line in ref.splitlines()])
        assert np.max(np.abs(vals)) > 0, fname


@pytest.mark.parametrize("mode", sorted(MODES), ids=[MODES[m][0][2:] for m in sorted(MODES)])
def test_fp32_mode_matches_reference(fdtd, mode):
    _need_ref()
    flag, comps, teta, phi, psi = MODES[mode]
    eps = _eps_map(mode, 100 + mode)
    kw = dict(mode=mode, size=_plane_shape(mode), use_pml=True, pml=3, use_tfsf=True, tfsf_left=5,
              tfsf_right=6, teta=teta, phi=phi, psi=psi)
    ref, _ = run_reference(materials={"eps": eps}, steps=40, **kw)
    assert sorted(ref) == sorted(comps)
    with fdtd.Simulation(materials={"eps": eps}, precision=fdtd.PREC_FP32, **kw) as sim:
        sim.step(40)
        got = {c: sim.field(c) for c in comps}
    for fam in ("E", "H"):
        names = [c for c in comps if c[0] == fam]
        num = sum(np.sum((got[c] - ref[c]) ** 2) for c in names)
        den = sum(np.sum(ref[c] ** 2) for c in names)
        assert den > 0
        assert np.sqrt(num / den) <= 1e-5, (fam, np.sqrt(num / den))


def test_exhy_1d_reproduces_reference_unit_test_vector(fdtd, monkeypatch):
    """The FP64 1-D ExHy mode through the C ABI against the golden vector of
    the reference's own unit test (Source/UnitTests/unit-test-internalscheme.cpp,
    test1D_ExHy, E_CENTERED; sine column): Ex after 200 steps, TF/SF 7 cells
    in from both ends of a 20-cell z axis, exact zeros in the scattered zone.
    The unit test sets dx, wavelength and Courant number as doubles, not
    through the command line's float parsing, so neither does this run."""
    import json

    monkeypatch.setattr(fdtd, "f32", float)

    g = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "exhy_1d_unit_test.json")))
    kw = dict(mode=fdtd.MODE_EXHY, size=(g["size"],), use_tfsf=True, tfsf_left=g["tfsf"], tfsf_right=g["tfsf"],
              dx=g["dx"], wavelength=g["wavelength"], courant=g["courant"], teta=0, phi=0, psi=90)
    with fdtd.Simulation(precision=fdtd.PREC_FP64_PLAIN, **kw) as sim:
        sim.step(g["steps"])
        ex = sim.field("Ex")
    assert ex.shape == (g["size"],)
    for k, (re, _im) in g["ex"].items():
        assert abs(ex[int(k)] - re) <= 1e-15, (k, ex[int(k)], re)
    assert ex[6] == 0.0 and ex[13] == 0.0


REF_COMPLEX = os.path.join(os.path.dirname(REF_BIN), "fdtd3d_complex")


def _write_complex_txt(path, arr):
    """Material TXT of the complex build: "coords re im" per line."""
    arr = np.asarray(arr, dtype=np.float64)
    idx = np.indices(arr.shape).reshape(arr.ndim, -1).T
    with open(path, "w") as f:
        for i, v in zip(idx, arr.reshape(-1)):
            f.write(" ".join(str(int(q)) for q in i) + " " + repr(float(v)) + " 0\n")


@pytest.mark.parametrize("mode,source", [(3, False), (6, True), (7, False)], ids=["3d", "2d-tez-source", "2d-tmx"])
def test_cli_complex_matches_reference_complex_build(fdtd, tmp_path, mode, source):
    """--complex-field-values (two runs: sine and cosine sources) writes the
    same "coords re im" TXT dumps as the reference's complex-field build."""
    if not os.path.exists(REF_COMPLEX):
        pytest.skip("complex reference binary not built")
    cli = os.path.join(os.path.dirname(fdtd.__file__), "fdtd3d-b200")
    if mode == 3:
        flags = ["--3d", "--size", "x:16,y:14,z:18", "--use-pml", "--pml-size", "x:3", "--same-size-pml",
                 "--use-tfsf", "--tfsf-size-left", "x:5", "--same-size-tfsf", "--tfsf-size-right", "x:5",
                 "--angle-teta", "30", "--angle-phi", "40", "--angle-psi", "10", "--time-steps", "25",
                 "--save-res", "--save-as-txt", "--manual-save-coords", "--save-start-coord", "x:0,y:0,z:0",
                 "--save-end-coord", "x:16,y:14,z:18"]
        shape = (16, 14, 18)
    else:
        flags = _flags(mode, 30, source)
        shape = _plane_shape(mode)
    eps = np.where(np.random.default_rng(mode).random(shape) < 0.3, 4.0, 1.0)
    _write_complex_txt(str(tmp_path / "eps.txt"), eps)
    flags += ["--load-eps-from-file", str(tmp_path / "eps.txt")]
    out = {}
    for name, exe, extra in (("ref", REF_COMPLEX, ["--use-ca-cb", "--use-ca-cb-pml"]),
                             ("b200", cli, ["--complex-field-values"])):
        d = tmp_path / name
        d.mkdir()
        r = subprocess.run([exe] + flags + extra, cwd=d, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
        out[name] = {f.name: f.read_text() for f in d.iterdir()}
    assert sorted(out["ref"]) == sorted(out["b200"]) and out["ref"]
    for fname, ref in out["ref"].items():
        mine = out["b200"][fname]
        assert len(ref.splitlines()[0].split()) == len(shape) + 2
        if mine != ref:
            diffs = [(a, b) for a, b in zip(ref.splitlines(), mine.splitlines()) if a != b]
            raise AssertionError(f"{fname}: {len(diffs)} lines differ, first: {diffs[:4]}")
        im = np.array([float(line.split()[-1]) for line in ref.splitlines()])
        assert np.max(np.abs(im)) > 0, fname


def test_cli_complex_materials_use_real_parts(fdtd, tmp_path):
    """Complex material files with nonzero imaginary parts: the reference's
    step reads the real part of every material value
    (Source/Layout/Approximation.cpp, Approximation::getMaterial), and so does
    --complex-field-values; TXT dumps byte-identical to the complex build."""
    if not os.path.exists(REF_COMPLEX):
        pytest.skip("complex reference binary not built")
    cli = os.path.join(os.path.dirname(fdtd.__file__), "fdtd3d-b200")
    flags = _flags(6, 30, False)
    shape = _plane_shape(6)
    rng = np.random.default_rng(11)
    eps = np.where(rng.random(shape) < 0.3, 4.0, 1.0)
    im = np.round(rng.uniform(-2, 2, shape), 3)
    idx = np.indices(shape).reshape(len(shape), -1).T
    with open(tmp_path / "eps.txt", "w") as f:
        for i, v, w in zip(idx, eps.reshape(-1), im.reshape(-1)):
            f.write(" ".join(str(int(q)) for q in i) + f" {float(v)!r} {float(w)!r}\n")
    flags += ["--load-eps-from-file", str(tmp_path / "eps.txt")]
    out = {}
    for name, exe, extra in (("ref", REF_COMPLEX, ["--use-ca-cb", "--use-ca-cb-pml"]),
                             ("b200", cli, ["--complex-field-values"])):
        d = tmp_path / name
        d.mkdir()
        r = subprocess.run([exe] + flags + extra, cwd=d, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
        out[name] = {f.name: f.read_text() for f in d.iterdir()}
    assert sorted(out["ref"]) == sorted(out["b200"]) and out["ref"]
    for fname, ref in out["ref"].items():
        assert out["b200"][fname] == ref, fname
