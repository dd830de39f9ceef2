"""Running DFT (fdtd_dft_setup / fdtd_dft_read) against a DFT accumulated
in numpy from the fields downloaded after every step, and FP32 against FP64
on a Drude slab (the metamaterial benchmark geometry, scaled down).

Bars: FP64 plain form against numpy <= 1e-12 relative L2 (both sum the same
FP64 values; the library compensates its sums); FP32 forms against numpy
from their own fields <= 1e-9; FP32 against FP64 on the slab <= 1e-4.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def numpy_dft(sim, comp, axis, index, freqs, steps, t_start, dt):
    acc = 0
    shift = 1.0 if comp.startswith("H") else 0.5
    for s in range(steps):
        sim.step(1)
        f = sim.field(comp)
        plane = np.take(f, index, axis=axis) if f.ndim == 3 else f
        t = (t_start + s + shift) * dt
        ph = np.exp(-2j * np.pi * np.asarray(freqs)[:, None, None] * t)
        acc = acc + plane[None] * ph
    return acc


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("prec,tol", [(0, 1e-12), (1, 1e-9)])
def test_dft_matches_numpy_accumulation(fdtd, prec, tol):
    kw = dict(mode=3, size=(20, 18, 24), use_pml=True, pml=3, use_tfsf=True, tfsf_left=5, tfsf_right=5,
              teta=30, phi=45, psi=20, precision=prec)
    freqs = [12e9, 15e9, 18e9]
    with fdtd.Simulation(**kw) as sim:
        dt = sim.scalars()["dt"]
        sim.dft_setup("Ey", 2, 17, freqs)
        ref = numpy_dft(sim, "Ey", 2, 17, freqs, 40, 0, dt)
        got = sim.dft()
    assert got.shape == ref.shape
    assert rel(got, ref) <= tol, rel(got, ref)


def test_dft_restart_and_h_component(fdtd):
    kw = dict(mode=2, size=(40, 36), use_pml=True, pml=5, point_source=(20, 18), point_source_mask=1 << 2,
              point_source_kind=1, point_source_bandwidth=0.5, teta=90, phi=0, psi=90, precision=0)
    with fdtd.Simulation(**kw) as sim:
        dt = sim.scalars()["dt"]
        sim.dft_setup("Hx", 2, 0, [15e9])
        sim.step(10)
        sim.dft_setup("Hx", 2, 0, [15e9])      # restart from zero at t = 10
        ref = numpy_dft(sim, "Hx", 2, 0, [15e9], 25, 10, dt)
        got = sim.dft()
    assert rel(got, ref) <= 1e-12


def test_dft_drude_slab_fp32_against_fp64(fdtd):
    """Drude slab (omega_p = 2 pi 30 GHz, gamma = 2 pi 1 GHz for eps and mu)
    normal to z, plane wave at normal incidence, PML; DFT of Ez at the
    slab's back face, FP32 against the FP64 plain form."""
    n = (16, 16, 64)
    z0, z1 = 26, 38
    om = np.zeros(n)
    ga = np.zeros(n)
    om[:, :, z0:z1] = np.float32(2 * np.pi * 30e9)
    ga[:, :, z0:z1] = np.float32(2 * np.pi * 1e9)
    mats = {"omegape": om, "gammae": ga, "omegapm": om, "gammam": ga}
    kw = dict(mode=3, size=n, use_pml=True, pml=(3, 3, 6), use_tfsf=True, tfsf_left=(4, 4, 10),
              tfsf_right=(4, 4, 10), teta=0, phi=0, psi=0, use_metamaterials=True)
    out = {}
    for prec in (0, 1):
        with fdtd.Simulation(materials=mats, precision=prec, **kw) as sim:
            sim.dft_setup("Ex", 2, z1, [15e9])
            sim.step(300)
            out[prec] = sim.dft()
    assert np.linalg.norm(out[0]) > 0
    assert rel(out[1], out[0]) <= 1e-4, rel(out[1], out[0])
