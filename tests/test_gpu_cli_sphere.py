"""The material-sphere flags of fdtd3d through fdtd3d-b200, byte-identical to
the reference CPU build: --eps-sphere / --mu-sphere / --omegape-sphere /
--omegapm-sphere with their -center and -radius flags, --sphere-accuracy and
--stair-sphere-approx (Source/Settings/Settings.inc.h:232-249), filled as
Scheme::initGrids does (Source/Scheme/Scheme.inc.h:2980-3160) by
Approximation::approximateSphereAccurate / approximateSphereStair
(Source/Layout/Approximation.cpp:387-764).  Each case writes the material
dumps (--save-materials) and the fields after the run; every file must match
the reference's byte for byte."""
import os
import subprocess

import pytest

from oracle.oracle import REF_BIN

pytestmark = pytest.mark.gpu

PML_TFSF = ["--use-pml", "--pml-size", "x:4", "--same-size-pml", "--use-tfsf", "--tfsf-size-left", "x:6",
            "--same-size-tfsf", "--tfsf-size-right", "x:6"]
CASES = {
    # the shape of the reference's Examples/sphere.txt, scaled down
    "3d_accurate": (["--3d", "--size", "x:24,y:22,z:20", "--angle-teta", "30", "--angle-phi", "40", "--angle-psi",
                     "10", "--eps-sphere", "4", "--eps-sphere-center", "x:12,y:11,z:10", "--eps-sphere-radius", "5"]
                    + PML_TFSF),
    "3d_stair_eps_mu": (["--3d", "--size", "x:22,y:20,z:24", "--angle-teta", "0", "--angle-phi", "0", "--angle-psi",
                         "0", "--stair-sphere-approx", "--eps-sphere", "2.5", "--eps-sphere-center", "x:11,y:9,z:12",
                         "--eps-sphere-radius", "6", "--mu-sphere", "1.5", "--mu-sphere-center", "x:10,y:10,z:11",
                         "--mu-sphere-radius", "4"] + PML_TFSF),
    "3d_accuracy_7_no_pml": ["--3d", "--size", "x:18,y:16,z:20", "--eps-sphere", "3.3", "--eps-sphere-center",
                             "x:9,y:7,z:10", "--eps-sphere-radius", "5", "--sphere-accuracy", "7",
                             "--point-source-ez", "--point-source", "x:4,y:8,z:10"],
    "3d_drude_omegape": (["--3d", "--size", "x:22,y:20,z:24", "--angle-teta", "0", "--angle-phi", "0",
                          "--angle-psi", "0", "--use-metamaterials", "--eps-sphere", "1.5", "--eps-sphere-center",
                          "x:11,y:10,z:12", "--eps-sphere-radius", "4", "--omegape-sphere", "0.8",
                          "--omegape-sphere-center", "x:11,y:10,z:12", "--omegape-sphere-radius", "3"] + PML_TFSF),
    "3d_double_material_precision": (["--3d", "--size", "x:18,y:16,z:20", "--angle-teta", "0", "--angle-phi", "0",
                                      "--angle-psi", "0", "--use-double-material-precision", "--eps-sphere", "4",
                                      "--eps-sphere-center", "x:9,y:8,z:10", "--eps-sphere-radius", "4"]
                                     + PML_TFSF),
    "tmz_accurate": ["--2d-tmz", "--size", "x:40,y:36", "--angle-teta", "90", "--angle-phi", "30", "--angle-psi",
                     "90", "--eps-sphere", "4", "--eps-sphere-center", "x:20,y:18", "--eps-sphere-radius", "9",
                     "--sphere-accuracy", "40"] + PML_TFSF,
    "3d_tfsf_right_zero": ["--3d", "--size", "x:22,y:20,z:24", "--angle-teta", "30", "--angle-phi", "40",
                           "--angle-psi", "10", "--eps-sphere", "4", "--eps-sphere-center", "x:11,y:10,z:12",
                           "--eps-sphere-radius", "5", "--use-pml", "--pml-size", "x:4", "--same-size-pml",
                           "--use-tfsf", "--tfsf-size-left", "x:6,y:6,z:7", "--tfsf-size-right", "x:0,y:6,z:0"],
    "exhy_accurate": ["--1d-exhy", "--size", "z:80", "--angle-teta", "0", "--angle-phi", "0", "--angle-psi", "0",
                      "--eps-sphere", "4", "--eps-sphere-center", "z:45", "--eps-sphere-radius", "12",
                      "--use-pml", "--pml-size", "z:6", "--use-tfsf", "--tfsf-size-left", "z:10",
                      "--tfsf-size-right", "z:0"],
}


def _run(exe, flags, d):
    d.mkdir()
    r = subprocess.run([exe] + flags, cwd=d, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    return {f.name: f.read_bytes() for f in d.iterdir()}


@pytest.mark.parametrize("case", sorted(CASES))
def test_cli_material_sphere_matches_reference(fdtd, tmp_path, case):
    if not os.path.exists(REF_BIN):
        pytest.skip("reference binary not built")
    flags = CASES[case] + ["--time-steps", "30", "--save-res", "--save-as-txt", "--save-materials"]
    ref = _run(REF_BIN, flags + ["--use-ca-cb", "--use-ca-cb-pml"], tmp_path / "ref")
    mine = _run(os.path.join(os.path.dirname(fdtd.__file__), "fdtd3d-b200"), flags, tmp_path / "b200")
    assert sorted(ref) == sorted(mine), (sorted(ref), sorted(mine))
    eps = [f for f in ref if "name=Eps" in f]
    assert eps and any(line.split()[-1] != b"1" for line in ref[eps[0]].splitlines()), "the sphere is in the dump"
    for name, data in ref.items():
        if mine[name] != data:
            a, b = data.decode().splitlines(), mine[name].decode().splitlines()
            diffs = [(x, y) for x, y in zip(a, b) if x != y]
            raise AssertionError(f"{case} {name}: {len(diffs)} of {len(a)} lines differ: {diffs[:3]}")
