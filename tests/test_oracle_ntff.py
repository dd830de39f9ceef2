"""Pins the NTFF restatement (oracle/ntff.py) to the reference's complex-field
build: the reference writes its NTFF files (--use-ntff) and, from two more runs
(T - 1 and T steps), its fields; the restatement evaluated on those fields
reproduces the printed values (six significant digits), for both layouts and
for the forward and the reverse diagram."""
import glob
import os
import subprocess
import tempfile

import numpy as np
import pytest

from oracle.ntff import ntff_values
from oracle.oracle import REF_BIN, f32

REF_COMPLEX = os.path.join(os.path.dirname(REF_BIN), "fdtd3d_complex")
N = (20, 18, 22)


def _flags(layout, steps):
    size = f"x:{N[0]},y:{N[1]},z:{N[2]}"
    return ["--3d", "--size", size, "--use-pml", "--pml-size", "x:3", "--same-size-pml",
            "--use-tfsf", "--tfsf-size-left", "x:6", "--same-size-tfsf", "--tfsf-size-right", "x:6",
            "--angle-teta", "30", "--angle-phi", "40", "--angle-psi", "10", "--time-steps", str(steps),
            "--layout-type", str(layout), "--use-ca-cb", "--use-ca-cb-pml"]


def _fields(tmp, layout, steps):
    d = os.path.join(tmp, f"f{layout}_{steps}")
    os.makedirs(d)
    size = f"x:{N[0]},y:{N[1]},z:{N[2]}"
    r = subprocess.run([REF_COMPLEX] + _flags(layout, steps) + [
        "--save-res", "--save-as-txt", "--manual-save-coords", "--save-start-coord", "x:0,y:0,z:0",
        "--save-end-coord", size], cwd=d, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    out = {}
    for comp in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
        (path,) = glob.glob(os.path.join(d, f"previous-1_*_[[]name={comp}].txt"))
        a = np.loadtxt(path)
        arr = np.zeros(N, dtype=complex)
        arr[a[:, 0].astype(int), a[:, 1].astype(int), a[:, 2].astype(int)] = a[:, 3] + 1j * a[:, 4]
        out[comp] = arr
    return out


@pytest.mark.skipif(not os.path.exists(REF_COMPLEX), reason="complex reference binary not built")
@pytest.mark.parametrize("layout,reverse", [(0, False), (1, False), (0, True)], ids=["e-fwd", "h-fwd", "e-rev"])
def test_ntff_restatement_matches_reference_files(layout, reverse):
    steps = 30
    with tempfile.TemporaryDirectory() as tmp:
        d = os.path.join(tmp, "ntff")
        os.makedirs(d)
        extra = ["--use-ntff", "--ntff-size", "x:4", "--same-size-ntff", "--interm-ntff-step", str(steps),
                 "--ntff-diff", "2"] + (["--ntff-reverse"] if reverse else [])
        r = subprocess.run([REF_COMPLEX] + _flags(layout, steps) + extra, cwd=d, capture_output=True, text=True,
                           timeout=300)
        assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
        cur = _fields(tmp, layout, steps)
        before = _fields(tmp, layout, steps - 1)
        h_prev = {c: before[c] for c in ("Hx", "Hy", "Hz")}
        teta = f32(30) * np.pi / 180.0
        for step in range(2):
            left = [4 + step] * 3
            right = [N[a] - 4 + 1 - step for a in range(3)]
            lines = open(os.path.join(d, f"ntff-res_[timestep={steps}]_[step={step}].txt")).read().splitlines()
            rows = [ln for ln in lines if ln.startswith("timestep = ")]
            if reverse:
                phis = [f32(40) * np.pi / 180.0]
            else:
                phis, a = [], 0.0
                while a <= 2 * np.pi + np.pi / 180:
                    phis.append(a)
                    a += np.pi * f32(10.0) / 180
            printed = [float(ln.split("angle NTFF = ")[1].split(",")[0]) for ln in rows]
            assert np.allclose(printed, phis, rtol=1e-5, atol=1e-6)
            ref = np.array([float(ln.split("NTFF value = ")[1]) for ln in rows])
            assert len(rows) == (1 if reverse else 37)
            # dx and the wavelength are the reference's defaults (double literals)
            mine = ntff_values(cur, h_prev, layout, left, right, 0.0005, 0.02, teta, phis)
            # the reference prints six significant digits, its angles too
            assert np.all(np.abs(mine - ref) <= 1e-5 * np.abs(ref) + 1e-300), (step, mine[:4], ref[:4])
            assert np.max(ref) > 0
