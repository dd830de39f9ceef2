"""Near-to-far-field transform on the device (fdtd_ntff, --use-ntff).

* fdtd3d-b200 --complex-field-values --use-ntff writes byte-identical NTFF
  files to the reference's complex-field build (oracle/_ref/fdtd3d_complex):
  forward and reverse diagrams, both layouts, two boxes (--ntff-diff 2), two
  save times, an odd-sized grid.
* fdtd_ntff agrees with the CPU restatement (oracle/ntff.py, itself pinned to
  the reference's files) to 1e-9 relative on the same fields.
* FP32 / FP16-storage runs (fdtd_keep_previous_level) give the FP64 form's
  values to the FP32 / FP16 bar, through the C ABI and through the CLI.
"""
import os
import subprocess

import numpy as np
import pytest

from oracle.ntff import ntff_values
from oracle.oracle import REF_BIN, write_material_txt

pytestmark = pytest.mark.gpu

REF_COMPLEX = os.path.join(os.path.dirname(REF_BIN), "fdtd3d_complex")

CASES = {
    "e_forward": ((20, 18, 22), 0, []),
    "h_forward": ((20, 18, 22), 1, []),
    "e_reverse": ((20, 18, 22), 0, ["--ntff-reverse"]),
    "h_reverse_odd": ((21, 19, 23), 1, ["--ntff-reverse"]),
    "e_odd_step_angle": ((21, 20, 19), 0, ["--ntff-step-angle", "7.5"]),
}


def _complex_txt(path, arr):
    arr = np.asarray(arr, dtype=np.float64)
    idx = np.indices(arr.shape).reshape(arr.ndim, -1).T
    with open(path, "w") as f:
        for i, v in zip(idx, arr.reshape(-1)):
            f.write(" ".join(str(int(q)) for q in i) + " " + repr(float(v)) + " 0\n")


@pytest.mark.parametrize("case", sorted(CASES))
def test_cli_ntff_matches_reference_complex_build(fdtd, tmp_path, case):
    if not os.path.exists(REF_COMPLEX):
        pytest.skip("complex reference binary not built")
    n, layout, extra = CASES[case]
    x, y, z = np.indices(n)
    eps = np.where((x - n[0] / 2) ** 2 + (y - n[1] / 2) ** 2 + (z - n[2] / 2) ** 2 < 12, 4.0, 1.0)
    _complex_txt(str(tmp_path / "eps.txt"), eps)
    size = f"x:{n[0]},y:{n[1]},z:{n[2]}"
    flags = ["--3d", "--size", size, "--use-pml", "--pml-size", "x:3", "--same-size-pml",
             "--use-tfsf", "--tfsf-size-left", "x:6", "--same-size-tfsf", "--tfsf-size-right", "x:6",
             "--angle-teta", "30", "--angle-phi", "40", "--angle-psi", "10", "--time-steps", "30",
             "--layout-type", str(layout), "--load-eps-from-file", str(tmp_path / "eps.txt"),
             "--use-ntff", "--ntff-size", "x:4", "--same-size-ntff", "--interm-ntff-step", "15",
             "--ntff-diff", "2"] + extra
    cli = os.path.join(os.path.dirname(fdtd.__file__), "fdtd3d-b200")
    out = {}
    for name, exe, more in (("ref", REF_COMPLEX, ["--use-ca-cb", "--use-ca-cb-pml"]),
                            ("b200", cli, ["--complex-field-values"])):
        d = tmp_path / name
        d.mkdir()
        r = subprocess.run([exe] + flags + more, cwd=d, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
        out[name] = {f.name: f.read_text() for f in d.iterdir()}
    assert sorted(out["ref"]) == sorted(out["b200"])
    assert len(out["ref"]) == 4, sorted(out["ref"])   # 2 save times x 2 boxes
    for fname, text in out["ref"].items():
        if out["b200"][fname] != text:
            diffs = [(a, b) for a, b in zip(text.splitlines(), out["b200"][fname].splitlines()) if a != b]
            raise AssertionError(f"{fname}: {len(diffs)} lines differ, first: {diffs[:4]}")


@pytest.mark.parametrize("layout", [0, 1])
def test_fdtd_ntff_matches_restatement(fdtd, layout):
    n = (24, 22, 26)
    kw = dict(mode=3, size=n, use_pml=True, pml=4, use_tfsf=True, tfsf_left=7, tfsf_right=7, teta=30, phi=40,
              psi=10, layout=layout)
    x, y, z = np.indices(n)
    eps = np.where((x - 12) ** 2 + (y - 11) ** 2 + (z - 13) ** 2 < 16, 4.0, 1.0)
    steps = 40

    def run(nsteps):
        sims = [fdtd.Simulation(precision=fdtd.PREC_FP64_PLAIN, source_phase=ph, materials={"eps": eps}, **kw)
                for ph in (0, 1)]
        for s in sims:
            s.step(nsteps)
        return sims

    before = run(steps - 1)
    h_prev = {c: before[0].field(c) + 1j * before[1].field(c) for c in ("Hx", "Hy", "Hz")}
    for s in before:
        s.close()
    sims = run(steps)
    cur = {c: sims[0].field(c) + 1j * sims[1].field(c) for c in fdtd.COMPONENTS}
    left, right = (5, 5, 5), (n[0] - 4, n[1] - 4, n[2] - 4)
    teta = fdtd.f32(30) * np.pi / 180.0
    phis = np.linspace(0, 2 * np.pi, 25)
    got = fdtd.ntff(sims[0], sims[1], left, right, teta, phis)
    want = ntff_values(cur, h_prev, layout, left, right, fdtd.f32(0.0005), fdtd.f32(0.02), teta, phis)
    for s in sims:
        s.close()
    assert np.all(want > 0)
    assert np.max(np.abs(got - want) / want) <= 1e-9, np.max(np.abs(got - want) / want)


def test_fdtd_ntff_rejects_what_it_does_not_provide(fdtd):
    kw = dict(mode=3, size=16, use_pml=True, pml=3)
    with fdtd.Simulation(precision=fdtd.PREC_FP32, **kw) as a, fdtd.Simulation(precision=fdtd.PREC_FP32,
                                                                            source_phase=1, **kw) as b:
        with pytest.raises(fdtd.FdtdError):
            fdtd.ntff(a, b, (4, 4, 4), (12, 12, 12), 0.5, [0.0])
    with fdtd.Simulation(**kw) as a, fdtd.Simulation(source_phase=1, **kw) as b:
        a.step(2)
        b.step(2)
        with pytest.raises(fdtd.FdtdError):
            fdtd.ntff(a, b, (0, 4, 4), (12, 12, 12), 0.5, [0.0])
        with pytest.raises(fdtd.FdtdError):
            fdtd.ntff(a, b, (4, 4, 4), (16, 12, 12), 0.5, [0.0])
        assert fdtd.ntff(a, b, (4, 4, 4), (12, 12, 12), 0.5, [0.0, 1.0]).shape == (2,)
    kw2 = dict(mode=2, size=(16, 16), use_pml=True, pml=3)
    with fdtd.Simulation(**kw2) as a, fdtd.Simulation(source_phase=1, **kw2) as b:
        with pytest.raises(fdtd.FdtdError):
            fdtd.ntff(a, b, (4, 4, 0), (12, 12, 1), 0.5, [0.0])


@pytest.mark.parametrize("layout,prec,steps", [(0, 1, 40), (0, 1, 41), (1, 1, 40), (0, 2, 40)])
def test_fdtd_ntff_fast_forms(fdtd, layout, prec, steps):
    """FP32 / FP16-storage runs with keep_previous_level against the FP64
    plain form's NTFF of the same configuration: relative difference per
    azimuth <= 1e-4 (FP32: the fields carry about 1e-6) and 2e-2 (FP16
    storage).  E_CENTERED takes the one-sweep path (pairs of steps, the
    last step of the call single), H_CENTERED the per-cell kernels (H copied
    before the last H update)."""
    n = (24, 22, 26)
    kw = dict(mode=3, size=n, use_pml=True, pml=4, use_tfsf=True, tfsf_left=7, tfsf_right=7, teta=30, phi=40,
              psi=10, layout=layout)
    x, y, z = np.indices(n)
    eps = np.where((x - 12) ** 2 + (y - 11) ** 2 + (z - 13) ** 2 < 16, 4.0, 1.0)
    left, right = (5, 5, 5), (n[0] - 4, n[1] - 4, n[2] - 4)
    teta = fdtd.f32(30) * np.pi / 180.0
    phis = np.linspace(0, 2 * np.pi, 25)
    vals = {}
    kernels = set()
    for p in (fdtd.PREC_FP64_PLAIN, prec):
        sims = [fdtd.Simulation(precision=p, source_phase=ph, materials={"eps": eps}, **kw) for ph in (0, 1)]
        try:
            for s in sims:
                s.keep_previous_level()
                s.step(steps // 2)
                s.step(steps - steps // 2)
                kernels.add(s.step_kernel)
            vals[p] = fdtd.ntff(sims[0], sims[1], left, right, teta, phis)
        finally:
            for s in sims:
                s.close()
    want, got = vals[fdtd.PREC_FP64_PLAIN], vals[prec]
    assert np.all(want > 0)
    err = np.max(np.abs(got - want) / want)
    assert err <= (1e-4 if prec == fdtd.PREC_FP32 else 2e-2), (err, kernels)
    assert "sweep2_tma" not in kernels   # every call ends on a single step


def test_cli_fp32_ntff_close_to_reference_complex_build(fdtd, tmp_path):
    """fdtd3d-b200 --precision fp32 --complex-field-values --use-ntff: the
    same NTFF files as the reference's complex build, values within 1e-4
    relative (the FP64 form writes them byte-identical)."""
    if not os.path.exists(REF_COMPLEX):
        pytest.skip("complex reference binary not built")
    n = (20, 18, 22)
    flags = ["--3d", "--size", f"x:{n[0]},y:{n[1]},z:{n[2]}", "--use-pml", "--pml-size", "x:3", "--same-size-pml",
             "--use-tfsf", "--tfsf-size-left", "x:6", "--same-size-tfsf", "--tfsf-size-right", "x:6",
             "--angle-teta", "30", "--angle-phi", "40", "--angle-psi", "10", "--time-steps", "30",
             "--use-ntff", "--ntff-size", "x:4", "--same-size-ntff", "--interm-ntff-step", "15"]
    cli = os.path.join(os.path.dirname(fdtd.__file__), "fdtd3d-b200")
    out = {}
    for name, exe, more in (("ref", REF_COMPLEX, ["--use-ca-cb", "--use-ca-cb-pml"]),
                            ("b200", cli, ["--complex-field-values", "--precision", "fp32"])):
        d = tmp_path / name
        d.mkdir()
        r = subprocess.run([exe] + flags + more, cwd=d, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
        out[name] = {f.name: f.read_text() for f in d.iterdir()}
    assert sorted(out["ref"]) == sorted(out["b200"]) and len(out["ref"]) == 2, sorted(out["b200"])
    for fname, text in out["ref"].items():
        a = [float(line.rsplit("=", 1)[1]) for line in text.splitlines() if "NTFF value" in line]
        b = [float(line.rsplit("=", 1)[1]) for line in out["b200"][fname].splitlines() if "NTFF value" in line]
        assert len(a) == len(b) > 10
        a, b = np.array(a), np.array(b)
        assert np.max(np.abs(b - a) / np.abs(a)) <= 1e-4, (fname, np.max(np.abs(b - a) / np.abs(a)))
