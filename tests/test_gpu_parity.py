"""Parity of the CUDA product (through the C ABI) against the oracle.

FP64 plain form: the bar is <= 1e-12 relative L2 per field (stated goal) and,
because the kernels keep the reference's operation order with --fmad=false,
the fields are expected to be bit-identical; both are asserted.
FP32 fused form: <= 1e-5 relative L2 of the E family and of the H family
against the FP64 oracle.  FP16-storage form: <= 2e-2 (10-bit mantissa).
"""
import json
import os

import numpy as np
import pytest

from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")

CASES = {
    "dim3_point_source": dict(mode=3, size=(14, 12, 16), point_source=(6, 5, 7), point_source_mask=(1 << 2) | (1 << 3),
                              teta=0, phi=0, psi=0),
    "dim3_tfsf_axis": dict(mode=3, size=16, use_tfsf=True, tfsf_left=4, tfsf_right=5, teta=0, phi=0, psi=0),
    "dim3_pml_tfsf_oblique": dict(mode=3, size=(18, 16, 20), use_pml=True, pml=(3, 4, 3), use_tfsf=True,
                                  tfsf_left=(5, 5, 6), tfsf_right=(6, 5, 5), teta=30, phi=45, psi=20),
    "dim3_pml_only": dict(mode=3, size=16, use_pml=True, pml=4, point_source=(8, 8, 8),
                          point_source_mask=1 << 1, teta=0, phi=0, psi=0),
    "dim3_drude": dict(mode=3, size=14, use_pml=True, pml=3, use_tfsf=True, tfsf_left=4, tfsf_right=4,
                       teta=0, phi=0, psi=0, use_metamaterials=True),
    "tmz_pml_tfsf": dict(mode=2, size=(40, 36), use_pml=True, pml=6, use_tfsf=True, tfsf_left=10, tfsf_right=9,
                         teta=90, phi=30, psi=90),
    "tmz_point_source": dict(mode=2, size=(33, 30), point_source=(15, 14), point_source_mask=1 << 2,
                             teta=90, phi=0, psi=90),
    # non-uniform mu and a point source on the outer shell take the per-cell
    # kernels of the fused forms instead of the one-sweep 3-D kernel
    "dim3_mu_per_cell": dict(mode=3, size=(15, 17, 14), use_pml=True, pml=3, use_tfsf=True, tfsf_left=5,
                             tfsf_right=5, teta=60, phi=20, psi=45),
    "dim3_boundary_source": dict(mode=3, size=14, point_source=(0, 7, 7), point_source_mask=1 << 1,
                                 teta=0, phi=0, psi=0),
    # one-sided TF/SF: a right size of 0 leaves those faces without terms
    "dim3_tfsf_right_zero": dict(mode=3, size=(18, 16, 20), use_pml=True, pml=3, use_tfsf=True, tfsf_left=(5, 5, 6),
                                 tfsf_right=(0, 5, 0), teta=30, phi=45, psi=20),
    "dim3_large_tiles": dict(mode=3, size=(40, 37, 70), use_pml=True, pml=(5, 4, 6), use_tfsf=True,
                             tfsf_left=(9, 8, 12), tfsf_right=(10, 9, 11), teta=30, phi=45, psi=0,
                             point_source=(20, 18, 35), point_source_mask=(1 << 0) | (1 << 5)),
}


def materials(name, shape):
    rng = np.random.default_rng(abs(hash(name)) % 2**32)
    if name == "dim3_pml_tfsf_oblique":
        x, y, z = np.indices(shape)
        return {"eps": np.where((x - 9) ** 2 + (y - 8) ** 2 + (z - 10) ** 2 < 12, 4.0, 1.0)}
    if name == "dim3_drude":
        om = np.zeros(shape)
        ga = np.zeros(shape)
        om[:, :, 6:9] = np.float32(2 * np.pi * 30e9)
        ga[:, :, 6:9] = np.float32(2 * np.pi * 1e9)
        return {"omegape": om, "gammae": ga, "omegapm": om, "gammam": ga}
    if name == "tmz_pml_tfsf":
        return {"eps": np.round(rng.uniform(1, 12, shape)).astype(np.float64)}
    if name == "dim3_mu_per_cell":
        return {"eps": np.round(rng.uniform(1, 6, shape)), "mu": np.round(rng.uniform(1, 3, shape))}
    if name == "dim3_large_tiles":
        x, y, z = np.indices(shape)
        return {"eps": np.where((x - 20) ** 2 + (y - 18) ** 2 + (z - 35) ** 2 < 64, 4.0, 1.0)}
    return None


def shape_of(kw):
    s = kw["size"]
    s = (s, s, s) if isinstance(s, int) else tuple(s)
    return s if kw["mode"] == 3 else s[:2]


def run_pair(fdtd, name, steps, precision):
    kw = CASES[name]
    shape = shape_of(kw)
    mats = materials(name, shape)
    o = Oracle(materials=mats, **kw)
    o.step(steps)
    sim = fdtd.Simulation(materials=mats, precision=precision, **kw)
    sim.step(steps)
    sim.sync()
    comps = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz") if kw["mode"] == 3 else ("Ez", "Hx", "Hy")
    out = {c: (sim.field(c), o.field(c)) for c in comps}
    sim.close()
    o.close()
    return out


def rel_l2(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / nb if nb > 0 else np.linalg.norm(a)


@pytest.mark.parametrize("name", sorted(CASES))
def test_plain_fp64_matches_oracle(fdtd, name):
    pairs = run_pair(fdtd, name, 24, fdtd.PREC_FP64_PLAIN)
    for comp, (g, r) in pairs.items():
        assert np.all(np.isfinite(g)), comp
        # per-field bar of the plain form, normalised by the dominant field of the family
        fam = [c for c in pairs if c[0] == comp[0]]
        scale = max(np.linalg.norm(pairs[c][1]) for c in fam)
        assert np.linalg.norm(g - r) <= 1e-12 * max(scale, 1e-300), (name, comp)
        # bit patterns, so that the sign of zero is compared too
        assert np.array_equal(g.view(np.int64), r.view(np.int64)), (name, comp, float(np.max(np.abs(g - r))))


def test_plain_fp64_config1_full(fdtd):
    """Config 1: 80^3, PML 10, TF/SF 15, theta = phi = psi = 0, 100 steps."""
    kw = dict(mode=3, size=80, use_pml=True, pml=10, use_tfsf=True, tfsf_left=15, tfsf_right=15,
              teta=0, phi=0, psi=0, dx=0.0005, wavelength=0.02, courant=0.5)
    o = Oracle(**kw)
    o.step(100)
    with fdtd.Simulation(precision=fdtd.PREC_FP64_PLAIN, **kw) as sim:
        sim.step(100)
        sim.sync()
        for comp in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
            g, r = sim.field(comp), o.field(comp)
            assert np.array_equal(g.view(np.int64), r.view(np.int64)), comp


@pytest.mark.parametrize("name", ["dim3_point_source", "dim3_tfsf_axis", "dim3_pml_tfsf_oblique",
                                  "dim3_pml_only", "tmz_pml_tfsf", "tmz_point_source", "dim3_mu_per_cell",
                                  "dim3_boundary_source", "dim3_large_tiles", "dim3_drude"])
@pytest.mark.parametrize("prec,tol", [(1, 1e-5), (2, 2e-2)])
def test_fused_forms_match_fp64(fdtd, name, prec, tol):
    pairs = run_pair(fdtd, name, 40, prec)
    for fam in ("E", "H"):
        cs = [c for c in pairs if c[0] == fam]
        g = np.concatenate([pairs[c][0].ravel() for c in cs])
        r = np.concatenate([pairs[c][1].ravel() for c in cs])
        assert np.all(np.isfinite(g))
        err = rel_l2(g, r)
        assert err <= tol, (name, prec, fam, err)


def test_energy_and_l2_reductions(fdtd):
    kw = CASES["dim3_pml_tfsf_oblique"]
    shape = shape_of(kw)
    mats = materials("dim3_pml_tfsf_oblique", shape)
    for prec in (0, 1):
        with fdtd.Simulation(materials=mats, precision=prec, **kw) as sim:
            sim.step(20)
            l2 = sim.reduce(fdtd.REDUCE_L2)
            energy = sim.reduce(fdtd.REDUCE_ENERGY)[0]
            f = {c: sim.field(c) for c in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")}
            eta0 = 376.730313461770655
            for k, c in enumerate(("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")):
                assert abs(l2[k] - np.sum(f[c] ** 2)) <= 1e-6 * np.sum(f[c] ** 2) + 1e-30, (prec, c)
            ref = sum(np.sum(mats["eps"] * f[c] ** 2) for c in ("Ex", "Ey", "Ez"))
            ref += sum(np.sum((eta0 * f[c]) ** 2) for c in ("Hx", "Hy", "Hz"))
            assert abs(energy - ref) <= 1e-5 * ref, (prec, energy, ref)


def test_upload_field_roundtrip_and_launch_count(fdtd):
    kw = dict(mode=3, size=(10, 11, 12))
    rng = np.random.default_rng(3)
    for prec in (0, 1, 2):
        with fdtd.Simulation(precision=prec, **kw) as sim:
            a = rng.standard_normal((10, 11, 12))
            sim.set_field("Ey", a)
            b = sim.field("Ey")
            tol = 0 if prec == 0 else (1e-7 if prec == 1 else 1e-3)
            assert np.max(np.abs(a - b)) <= tol * np.max(np.abs(a)) + 0.0
            n0 = sim.launch_count()
            sim.step(3)
            sim.sync()
            assert sim.launch_count() > n0


def test_sync_with_timeout_returns(fdtd):
    with fdtd.Simulation(mode=3, size=24, precision=1) as sim:
        sim.step(5)
        sim.sync(timeout_ns=10_000_000_000)


def test_unsupported_combination_is_reported(fdtd):
    # double material precision with metamaterials: the reference's
    # eight-point Drude average is unreachable (Approximation.cpp:167-197)
    with pytest.raises(fdtd.FdtdError):
        fdtd.Simulation(mode=3, size=(12, 12, 12), use_pml=True, pml=2, use_metamaterials=True,
                        double_material_precision=True, precision=1)


def test_cli_dropin_matches_reference_txt(fdtd, tmp_path):
    """fdtd3d-b200 takes the reference's flags and writes the same TXT dumps as
    the reference CPU build (oracle/_ref/fdtd3d) for the same run."""
    import subprocess

    from oracle.oracle import REF_BIN

    if not os.path.exists(REF_BIN):
        pytest.skip("reference binary not built")
    cli = os.path.join(os.path.dirname(fdtd.__file__), "fdtd3d-b200")
    flags = ["--3d", "--size", "x:18,y:16,z:20", "--use-pml", "--pml-size", "x:3", "--same-size-pml",
             "--use-tfsf", "--tfsf-size-left", "x:5", "--same-size-tfsf", "--tfsf-size-right", "x:5",
             "--angle-teta", "30", "--angle-phi", "45", "--angle-psi", "10", "--dx", "0.0005",
             "--wavelength", "0.02", "--courant-factor", "0.5", "--time-steps", "25", "--save-res",
             "--save-as-txt", "--manual-save-coords", "--save-start-coord", "x:0,y:0,z:0",
             "--save-end-coord", "x:18,y:16,z:20"]
    out = {}
    for name, exe, extra in (("ref", REF_BIN, ["--use-ca-cb", "--use-ca-cb-pml"]), ("b200", cli, [])):
        d = tmp_path / name
        d.mkdir()
        r = subprocess.run([exe] + flags + extra, cwd=d, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stdout + r.stderr
        assert "Total time = " in r.stdout
        out[name] = {f.name: f.read_text() for f in d.iterdir()}
    assert sorted(out["ref"]) == sorted(out["b200"])
    for fname, text in out["ref"].items():
        mine = out["b200"][fname]
        if mine != text:
            diffs = [(a, b) for a, b in zip(text.splitlines(), mine.splitlines()) if a != b]
            raise AssertionError(f"{fname}: {len(diffs)} lines differ, first: {diffs[:4]}")


def test_cli_dat_output_and_material_files(fdtd, tmp_path):
    """--save-as-dat writes the values of the TXT dump as raw FP64 (z fastest)
    under the same name with .dat; a permittivity map gives the same run from
    a .txt file (the reference's TXT loader) and from a .dat file (raw FP64);
    a partial save region is the matching sub-block; a .dat of the wrong size
    and an unknown extension are refused."""
    import subprocess

    from oracle.oracle import write_material_txt

    cli = os.path.join(os.path.dirname(fdtd.__file__), "fdtd3d-b200")
    n = (14, 12, 16)
    rng = np.random.default_rng(7)
    eps = np.where(rng.random(n) < 0.3, 4.0, 1.0)   # exact in FP32, as the TXT loader's stof keeps it
    write_material_txt(str(tmp_path / "eps.txt"), eps)
    eps.astype(np.float64).tofile(str(tmp_path / "eps.dat"))
    eps[:2].astype(np.float64).tofile(str(tmp_path / "short.dat"))
    (tmp_path / "eps.bin").write_bytes(b"")
    flags = ["--3d", "--size", "x:14,y:12,z:16", "--use-pml", "--pml-size", "x:2", "--same-size-pml",
             "--use-tfsf", "--tfsf-size-left", "x:4", "--same-size-tfsf", "--tfsf-size-right", "x:4",
             "--angle-teta", "30", "--angle-phi", "45", "--angle-psi", "10", "--time-steps", "15",
             "--save-res", "--save-as-txt", "--save-as-dat", "--manual-save-coords"]
    full = ["--save-start-coord", "x:0,y:0,z:0", "--save-end-coord", "x:14,y:12,z:16"]
    part = ["--save-start-coord", "x:1,y:2,z:3", "--save-end-coord", "x:10,y:9,z:11"]

    def run(name, mat, region, ok=True):
        d = tmp_path / name
        d.mkdir()
        r = subprocess.run([cli] + flags + region + ["--load-eps-from-file", str(tmp_path / mat)], cwd=d,
                           capture_output=True, text=True, timeout=300)
        assert (r.returncode == 0) == ok, r.stdout + r.stderr
        return d

    a, b, c = run("txt", "eps.txt", full), run("dat", "eps.dat", full), run("part", "eps.txt", part)
    run("short", "short.dat", full, ok=False)
    run("ext", "eps.bin", full, ok=False)
    for comp in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
        name = f"previous-1_[timestep=15]_[pid=0]_[name={comp}]"
        va = np.fromfile(str(a / (name + ".dat")), dtype=np.float64)
        assert va.size == np.prod(n)
        assert (b / (name + ".dat")).read_bytes() == (a / (name + ".dat")).read_bytes(), comp
        txt = np.array([float(line.split()[3]) for line in (a / (name + ".txt")).read_text().splitlines()])
        scale = max(np.max(np.abs(va)), 1e-300)
        assert np.max(np.abs(txt - va)) <= 1e-14 * scale, comp
        vp = np.fromfile(str(c / (name + ".dat")), dtype=np.float64)
        assert np.array_equal(vp, va.reshape(n)[1:10, 2:9, 3:11].reshape(-1)), comp
