"""The dump options of Scheme::saveGrids through fdtd3d-b200, byte-identical
to the reference CPU builds (Source/Scheme/Scheme.inc.h:4113-4530,
Source/Scheme/SchemeHelper.h:100-120): intermediate dumps
(--save-interm-res, --interm-save-step), the scattered field
(--save-scattered-field-res, --save-scattered--field-interm), the 1-D
incident grids (--save-tfsf-e-incident, --save-tfsf-h-incident), the save
region without the PML (--save-no-pml) and across another orthogonal axis
(--orth-axis-x / -y)."""
import os
import subprocess

import pytest

from oracle.oracle import REF_BIN

pytestmark = pytest.mark.gpu

REF_COMPLEX = os.path.join(os.path.dirname(REF_BIN), "fdtd3d_complex")
TFSF = ["--use-tfsf", "--tfsf-size-left", "x:5", "--same-size-tfsf", "--tfsf-size-right", "x:5",
        "--angle-teta", "30", "--angle-phi", "40", "--angle-psi", "10"]

CASES = {
    "3d_interm_scattered_incident": (["--3d", "--size", "x:16,y:14,z:18"] + TFSF +
                                     ["--save-interm-res", "--interm-save-step", "10", "--save-scattered-field-res",
                                      "--save-scattered--field-interm", "--save-tfsf-e-incident",
                                      "--save-tfsf-h-incident"]),
    "3d_h_centered_scattered": (["--3d", "--size", "x:16,y:14,z:18", "--layout-type", "1"] + TFSF +
                                ["--save-scattered-field-res"]),
    "3d_no_pml_orth_x": ["--3d", "--size", "x:16,y:14,z:18", "--save-no-pml", "--orth-axis-x"] + TFSF,
    "3d_orth_y_interm": (["--3d", "--size", "x:16,y:14,z:18", "--orth-axis-y", "--save-interm-res",
                          "--interm-save-step", "8"] + TFSF),
    "tmz_no_pml_scattered": (["--2d-tmz", "--size", "x:24,y:20", "--save-no-pml", "--save-scattered-field-res",
                              "--use-tfsf", "--tfsf-size-left", "x:6", "--same-size-tfsf", "--tfsf-size-right",
                              "x:6", "--angle-teta", "90", "--angle-phi", "30", "--angle-psi", "90"]),
    "eyhz_no_pml_interm": (["--1d-eyhz", "--size", "x:40", "--save-no-pml", "--save-interm-res",
                            "--interm-save-step", "12", "--save-tfsf-e-incident", "--use-tfsf", "--tfsf-size-left",
                            "x:8", "--same-size-tfsf", "--tfsf-size-right", "x:8", "--angle-teta", "90",
                            "--angle-phi", "0", "--angle-psi", "0"]),
}


def _run_pair(fdtd, ref_bin, flags, tmp_path, extra_ours=()):
    cli = os.path.join(os.path.dirname(fdtd.__file__), "fdtd3d-b200")
    out = {}
    for name, exe, more in (("ref", ref_bin, ["--use-ca-cb", "--use-ca-cb-pml"]), ("b200", cli, list(extra_ours))):
        d = tmp_path / name
        d.mkdir()
        r = subprocess.run([exe] + flags + more, cwd=d, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
        out[name] = {f.name: f.read_bytes() for f in d.iterdir()}
    return out


def _compare(out, min_files):
    assert sorted(out["ref"]) == sorted(out["b200"]), (sorted(out["ref"]), sorted(out["b200"]))
    assert len(out["ref"]) >= min_files, sorted(out["ref"])
    for fname, data in out["ref"].items():
        if out["b200"][fname] != data:
            if fname.endswith(".txt"):
                a, b = data.decode().splitlines(), out["b200"][fname].decode().splitlines()
                diffs = [(x, y) for x, y in zip(a, b) if x != y]
                raise AssertionError(f"{fname}: {len(a)} vs {len(b)} lines, {len(diffs)} differ: {diffs[:3]}")
            raise AssertionError(f"{fname} differs")


@pytest.mark.parametrize("case", sorted(CASES))
def test_cli_dump_options_match_reference(fdtd, tmp_path, case):
    if not os.path.exists(REF_BIN):
        pytest.skip("reference binary not built")
    flags = CASES[case] + ["--use-pml", "--pml-size", "x:3", "--same-size-pml", "--time-steps", "25", "--save-res",
                           "--save-as-txt"]
    _compare(_run_pair(fdtd, REF_BIN, flags, tmp_path), 2)


def test_cli_complex_interm_scattered_match_reference(fdtd, tmp_path):
    if not os.path.exists(REF_COMPLEX):
        pytest.skip("complex reference binary not built")
    flags = CASES["3d_interm_scattered_incident"] + ["--use-pml", "--pml-size", "x:3", "--same-size-pml",
                                                     "--time-steps", "25", "--save-res", "--save-as-txt"]
    _compare(_run_pair(fdtd, REF_COMPLEX, flags, tmp_path, ["--complex-field-values"]), 2)


def _material_txt(path, shape, seed, imag=False):
    import numpy as np

    rng = np.random.default_rng(seed)
    v = np.where(rng.random(shape) < 0.3, 4.0, 1.0)
    w = np.round(rng.uniform(-1, 1, shape), 3)
    idx = np.indices(shape).reshape(len(shape), -1).T
    with open(path, "w") as f:
        for i, a, b in zip(idx, v.reshape(-1), w.reshape(-1)):
            f.write(" ".join(str(int(q)) for q in i) + f" {float(a)!r}" + (f" {float(b)!r}" if imag else "") + "\n")


@pytest.mark.parametrize("variant", ["3d", "3d_meta_no_pml", "tmz_manual", "3d_dmp", "complex"])
def test_cli_save_materials_matches_reference(fdtd, tmp_path, variant):
    ref = REF_COMPLEX if variant == "complex" else REF_BIN
    if not os.path.exists(ref):
        pytest.skip("reference binary not built")
    if variant == "tmz_manual":
        flags = ["--2d-tmz", "--size", "x:20,y:18", "--manual-save-coords", "--save-start-coord", "x:2,y:3",
                 "--save-end-coord", "x:15,y:11"]
        shape = (20, 18)
    else:
        flags = ["--3d", "--size", "x:12,y:10,z:14"]
        shape = (12, 10, 14)
    if variant == "3d_dmp":
        flags.append("--use-double-material-precision")
        shape = tuple(2 * s for s in shape)
    _material_txt(str(tmp_path / "eps.txt"), shape, 4, imag=variant == "complex")
    flags += ["--use-pml", "--pml-size", "x:2", "--same-size-pml", "--time-steps", "4", "--save-res", "--save-as-txt",
              "--save-materials", "--load-eps-from-file", str(tmp_path / "eps.txt")]
    if variant == "3d_meta_no_pml":
        flags += ["--use-metamaterials", "--save-no-pml"]
    out = _run_pair(fdtd, ref, flags, tmp_path, ["--complex-field-values"] if variant == "complex" else [])
    _compare(out, 4)
    assert any("name=Eps" in f for f in out["ref"])
