"""J / M current sources (--current-source, --current-source-jx .. -mz).

After the curl update of a component with a current source, its cell takes
-= I dx Cb, I = sin(w t) mu0 / dt / 2 at the component's time (t on E,
t + 1/2 on H), before D -> E (Source/Scheme/Scheme.inc.h:1171-1260,
Source/Scheme/InternalScheme.inc.h:792-795, 2423-2449).  The complex-field
build drives cos(w (t - 1)) - i sin(w (t - 1)) instead.

* fdtd3d-b200 and the reference CPU build write byte-identical TXT dumps for
  current sources in 3-D (with PML, with TF/SF, in both layouts), in 2-D and
  in 1-D modes, and on the outer shell (where the reference's precomputed Cb
  is zero, so the source does nothing).
* --complex-field-values matches the reference's complex-field build.
* The FP32 per-cell form agrees with the FP64 form to 2e-5 relative L2.
"""
import os
import subprocess

import numpy as np
import pytest

from oracle.oracle import REF_BIN, write_material_txt

pytestmark = pytest.mark.gpu

REF_COMPLEX = os.path.join(os.path.dirname(REF_BIN), "fdtd3d_complex")
NAMES = ("x", "y", "z")

# name: (mode flag, kept axes, size, current cell, current flags, extra flags)
CASES = {
    "3d_pml": ("--3d", (0, 1, 2), (16, 14, 18), (8, 7, 9), ["jz", "my"], []),
    "3d_pml_tfsf": ("--3d", (0, 1, 2), (16, 14, 18), (7, 6, 8), ["jx", "jy", "mz"],
                    ["--use-tfsf", "--tfsf-size-left", "x:5", "--same-size-tfsf", "--tfsf-size-right", "x:5",
                     "--angle-teta", "30", "--angle-phi", "40", "--angle-psi", "10"]),
    "3d_h_centered": ("--3d", (0, 1, 2), (16, 14, 18), (8, 7, 9), ["jy", "mx"], ["--layout-type", "1"]),
    "3d_shell": ("--3d", (0, 1, 2), (16, 14, 18), (0, 7, 9), ["jz", "my"], []),
    "tmz": ("--2d-tmz", (0, 1), (30, 26, 1), (12, 11, 0), ["jz", "mx"], []),
    "tez": ("--2d-tez", (0, 1), (30, 26, 1), (14, 10, 0), ["jx", "mz"], []),
    "tex": ("--2d-tex", (1, 2), (1, 24, 28), (0, 12, 13), ["jy", "mx"], []),
    "exhy": ("--1d-exhy", (2,), (1, 1, 60), (0, 0, 29), ["jx", "my"], []),
}


def _flags(case, steps=25):
    flag, kept, size, cell, cur, extra = CASES[case]
    sz = ",".join(f"{NAMES[a]}:{size[a]}" for a in kept)
    return ([flag, "--size", sz, "--use-pml", "--pml-size", "x:3", "--same-size-pml", "--time-steps", str(steps),
             "--current-source", ",".join(f"{NAMES[a]}:{cell[a]}" for a in kept)]
            + [f"--current-source-{c}" for c in cur] + extra
            + ["--save-res", "--save-as-txt", "--manual-save-coords",
               "--save-start-coord", ",".join(f"{NAMES[a]}:0" for a in kept), "--save-end-coord", sz])


def _eps(case):
    _, kept, size, _, _, _ = CASES[case]
    shape = tuple(size[a] for a in kept)
    return np.where(np.random.default_rng(len(case)).random(shape) < 0.3, 3.0, 1.0)


def _run(exe, flags, d):
    d.mkdir()
    r = subprocess.run([exe] + flags, cwd=d, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    return {f.name: f.read_text() for f in d.iterdir()}


def _compare(ref, mine):
    assert sorted(ref) == sorted(mine) and ref
    for fname, text in ref.items():
        if mine[fname] != text:
            diffs = [(a, b) for a, b in zip(text.splitlines(), mine[fname].splitlines()) if a != b]
            raise AssertionError(f"{fname}: {len(diffs)} lines differ, first: {diffs[:4]}")


@pytest.mark.parametrize("case", sorted(CASES))
def test_cli_current_source_matches_reference_txt(fdtd, tmp_path, case):
    if not os.path.exists(REF_BIN):
        pytest.skip("reference binary not built")
    cli = os.path.join(os.path.dirname(fdtd.__file__), "fdtd3d-b200")
    write_material_txt(str(tmp_path / "eps.txt"), _eps(case))
    flags = _flags(case) + ["--load-eps-from-file", str(tmp_path / "eps.txt")]
    ref = _run(REF_BIN, flags + ["--use-ca-cb", "--use-ca-cb-pml"], tmp_path / "ref")
    mine = _run(cli, flags, tmp_path / "b200")
    _compare(ref, mine)
    # the source must be seen (except on the shell, where it does nothing)
    peak = max(max(abs(float(line.split()[-1])) for line in t.splitlines()) for t in ref.values())
    if case == "3d_shell":
        assert peak == 0.0
    else:
        assert peak > 0.0


def test_cli_complex_current_source_matches_reference_complex_build(fdtd, tmp_path):
    if not os.path.exists(REF_COMPLEX):
        pytest.skip("complex reference binary not built")
    cli = os.path.join(os.path.dirname(fdtd.__file__), "fdtd3d-b200")
    flags = _flags("3d_pml_tfsf", 20)
    ref = _run(REF_COMPLEX, flags + ["--use-ca-cb", "--use-ca-cb-pml"], tmp_path / "ref")
    mine = _run(cli, flags + ["--complex-field-values"], tmp_path / "b200")
    _compare(ref, mine)


@pytest.mark.parametrize("layout,mask,pos,nz,want", [
    (0, (1 << 2) | (1 << 4), (11, 10, 13), 28, "sweep3d_tma"),     # the TMA sweep + the current fix-up
    (0, (1 << 0) | (1 << 1) | (1 << 5), (12, 9, 14), 28, "sweep3d_tma"),
    (0, (1 << 2) | (1 << 4), (11, 10, 13), 26, "fused3d_regblock"),   # the register-blocked sweep + fix-up
    (0, (1 << 2) | (1 << 4), (4, 10, 13), 28, "per_cell"),         # next to the PML: the per-cell kernels
    (1, (1 << 2) | (1 << 4), (11, 10, 13), 28, "per_cell")])       # H_CENTERED: the per-cell kernels
def test_fp32_current_source_matches_fp64(fdtd, layout, mask, pos, nz, want):
    """J / M currents in the FP32 forms against the FP64 plain form.  In 3-D
    E_CENTERED with the cell and its neighbours outside the PML, the
    one-sweep kernel runs every step and the current enters as the step's
    linear response (launch_current_fix); otherwise the per-cell kernels,
    which fold it into the curl."""
    kw = dict(mode=3, size=(24, 22, nz), use_pml=True, pml=4, current_source=pos,
              current_source_mask=mask, layout=layout)
    out = {}
    for prec in (fdtd.PREC_FP64_PLAIN, fdtd.PREC_FP32):
        with fdtd.Simulation(precision=prec, **kw) as sim:
            sim.step(40)
            out[prec] = {c: sim.field(c) for c in fdtd.COMPONENTS}
            if prec == fdtd.PREC_FP32:
                assert sim.step_kernel == want, sim.step_kernel
    for fam in ("E", "H"):
        names = [c for c in fdtd.COMPONENTS if c[0] == fam]
        num = sum(np.sum((out[1][c] - out[0][c]) ** 2) for c in names)
        den = sum(np.sum(out[0][c] ** 2) for c in names)
        assert den > 0
        # a point current concentrates the field on a few cells around it, where
        # FP32 rounding accumulates over the run: 2e-5 (plane-wave runs hold 1e-5)
        assert np.sqrt(num / den) <= 2e-5, (fam, np.sqrt(num / den))
