"""Python handle on the oracle (test infrastructure only).

Two checkers live here, and nothing in the product imports this module:

* ``Oracle`` wraps ``oracle/_ref/liboracle.so``, the project's plain-C
  restatement of the fdtd3d leapfrog step (``oracle/fdtd_oracle.c``).
* ``run_reference`` runs ``oracle/_ref/fdtd3d``, the unmodified reference CPU
  solver compiled from its own sources by ``oracle/Makefile``, and parses the
  ``--save-as-txt`` dumps it writes (``Source/File-Management/Dumper/TXTDumper.h``;
  15 significant digits, z fastest).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may use it, and only as the checker / the timed CPU baseline.
"""
from __future__ import annotations

import ctypes
import glob
import os
import struct
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
LIB_PATH = os.path.join(REF_DIR, "liboracle.so")
REF_BIN = os.path.join(REF_DIR, "fdtd3d")
# the reference built with its own CUDA path (oracle/Makefile target ref_cuda)
REF_CUDA_BIN = os.path.join(os.path.dirname(REF_BIN), "fdtd3d_cuda")

COMPONENTS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
MATERIALS = ("eps", "mu", "omegape", "omegapm", "gammae", "gammam")


def f32(x: float) -> float:
    """Round like std::stof: the reference parses float flags to float."""
    return struct.unpack("f", struct.pack("f", float(x)))[0]


class _Cfg(ctypes.Structure):
    _fields_ = [
        ("mode", ctypes.c_int),
        ("size", ctypes.c_int * 3),
        ("pml", ctypes.c_int * 3),
        ("tfsf_left", ctypes.c_int * 3),
        ("tfsf_right", ctypes.c_int * 3),
        ("dx", ctypes.c_double),
        ("wavelength", ctypes.c_double),
        ("courant", ctypes.c_double),
        ("angle_teta", ctypes.c_double),
        ("angle_phi", ctypes.c_double),
        ("angle_psi", ctypes.c_double),
        ("use_pml", ctypes.c_int),
        ("use_tfsf", ctypes.c_int),
        ("use_metamaterials", ctypes.c_int),
        ("point_source", ctypes.c_int * 3),
        ("point_source_mask", ctypes.c_int),
        ("skip_first_update", ctypes.c_int),
        ("point_source_kind", ctypes.c_int),
        ("point_source_bandwidth", ctypes.c_double),
    ]


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-C", HERE, "oracle"], check=True, capture_output=True)
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.fdtd_oracle_create.restype = ctypes.c_void_p
        _lib.fdtd_oracle_create.argtypes = [ctypes.POINTER(_Cfg), ctypes.POINTER(ctypes.c_void_p)]
        _lib.fdtd_oracle_destroy.argtypes = [ctypes.c_void_p]
        _lib.fdtd_oracle_step.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32]
        _lib.fdtd_oracle_get.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        _lib.fdtd_oracle_get.restype = ctypes.c_int
        _lib.fdtd_oracle_scalars.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        _lib.fdtd_oracle_incident.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        _lib.fdtd_oracle_exhy_1d.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                             ctypes.c_double, ctypes.c_double, ctypes.c_uint32,
                                             ctypes.c_void_p, ctypes.c_void_p]
    return _lib


def _triple(v, default):
    if v is None:
        return (default,) * 3
    if isinstance(v, (int, np.integer)):
        return (int(v),) * 3
    v = tuple(int(a) for a in v)
    return v + (default,) * (3 - len(v))


class Oracle:
    """One simulation of the restated step; arrays are x-major, z fastest."""

    def __init__(self, *, mode=3, size=(20, 20, 20), pml=None, tfsf_left=None, tfsf_right=None,
                 dx=0.0005, wavelength=0.02, courant=0.5, teta=90.0, phi=0.0, psi=90.0,
                 use_pml=False, use_tfsf=False, use_metamaterials=False,
                 point_source=(0, 0, 0), point_source_mask=0, skip_first_update=True,
                 point_source_kind=0, point_source_bandwidth=0.0, materials=None, precision=None):
        c = _Cfg()
        c.mode = mode
        size = _triple(size, 1)
        if mode == 2:
            size = (size[0], size[1], 1)
        c.size[:] = size
        c.pml[:] = _triple(pml, 0)
        c.tfsf_left[:] = _triple(tfsf_left, 0)
        c.tfsf_right[:] = _triple(tfsf_right, 0)
        c.dx, c.wavelength, c.courant = f32(dx), f32(wavelength), f32(courant)
        c.angle_teta, c.angle_phi, c.angle_psi = f32(teta), f32(phi), f32(psi)
        c.use_pml, c.use_tfsf, c.use_metamaterials = int(use_pml), int(use_tfsf), int(use_metamaterials)
        c.point_source[:] = _triple(point_source, 0)
        c.point_source_mask = point_source_mask
        c.skip_first_update = int(skip_first_update)
        c.point_source_kind = int(point_source_kind)
        c.point_source_bandwidth = float(point_source_bandwidth)
        self.cfg = c
        self.shape = (size[0], size[1], size[2]) if mode == 3 else (size[0], size[1])
        self.n = int(np.prod(self.shape))
        self._keep = []
        ptrs = (ctypes.c_void_p * 6)()
        for i, name in enumerate(MATERIALS):
            arr = None if materials is None else materials.get(name)
            if arr is not None:
                a = np.ascontiguousarray(arr, dtype=np.float64).reshape(-1)
                assert a.size == self.n
                self._keep.append(a)
                ptrs[i] = a.ctypes.data
        self._h = lib().fdtd_oracle_create(ctypes.byref(c), ptrs)
        if not self._h:
            raise MemoryError("oracle allocation failed")
        self.t = 0

    def step(self, n: int) -> None:
        lib().fdtd_oracle_step(self._h, self.t, n)
        self.t += n

    def field(self, comp, level: int = 1) -> np.ndarray:
        k = COMPONENTS.index(comp) if isinstance(comp, str) else comp
        out = np.empty(self.n, dtype=np.float64)
        if lib().fdtd_oracle_get(self._h, k, level, out.ctypes.data) != 0:
            raise KeyError(comp)
        return out.reshape(self.shape)

    def scalars(self):
        out = np.empty(3, dtype=np.float64)
        lib().fdtd_oracle_scalars(self._h, out.ctypes.data)
        return {"dt": out[0], "frequency": out[1], "rel_phase_velocity": out[2]}

    def incident(self):
        m = 500 * self.shape[0]
        e = np.empty(m)
        h = np.empty(m)
        lib().fdtd_oracle_incident(self._h, e.ctypes.data, h.ctypes.data)
        return e, h

    def close(self):
        if self._h:
            lib().fdtd_oracle_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def exhy_1d(size=20, tfsf=7, dx=0.002, wavelength=0.2, courant=0.5, steps=200):
    s = np.empty(size)
    c = np.empty(size)
    lib().fdtd_oracle_exhy_1d(size, tfsf, dx, wavelength, courant, steps, s.ctypes.data, c.ctypes.data)
    return s, c


# --------------------------------------------------------------------------
# reference binary


def write_material_txt(path: str, arr: np.ndarray) -> None:
    """TXT grid in the reference loader's layout: 'x y [z] value', z fastest."""
    arr = np.asarray(arr, dtype=np.float64)
    idx = np.indices(arr.shape).reshape(arr.ndim, -1).T
    vals = arr.reshape(-1)
    with open(path, "w") as f:
        for i, v in zip(idx, vals):
            f.write(" ".join(str(int(q)) for q in i) + " " + repr(float(v)) + "\n")


# reference mode flags (Source/Settings/Settings.inc.h:48-60) and the axes
# each mode keeps
MODE_FLAGS = {2: "--2d-tmz", 3: "--3d", 4: "--2d-tex", 5: "--2d-tey", 6: "--2d-tez", 7: "--2d-tmx", 8: "--2d-tmy",
              10: "--1d-exhy", 11: "--1d-exhz", 12: "--1d-eyhx", 13: "--1d-eyhz", 14: "--1d-ezhx", 15: "--1d-ezhy"}
MODE_KEPT = {2: (0, 1), 3: (0, 1, 2), 4: (1, 2), 5: (0, 2), 6: (0, 1), 7: (1, 2), 8: (0, 2),
             10: (2,), 11: (1,), 12: (2,), 13: (0,), 14: (1,), 15: (0,)}


def mode_axes(mode):
    """The axes a mode keeps (x, y, z order)."""
    return MODE_KEPT[mode]


def _plane(v, mode, default):
    """Per-axis triple of a mode: a sequence as long as the kept axes gives
    those axes of a 2-D or 1-D mode."""
    axes = mode_axes(mode)
    if v is not None and not isinstance(v, (int, np.integer)) and len(v) == len(axes) and len(axes) < 3:
        t = [default] * 3
        for a, val in zip(axes, v):
            t[a] = int(val)
        return tuple(t)
    return _triple(v, default)


def reference_args(*, mode=3, size=(20, 20, 20), pml=None, tfsf_left=None, tfsf_right=None,
                   dx=0.0005, wavelength=0.02, courant=0.5, teta=90.0, phi=0.0, psi=90.0,
                   use_pml=False, use_tfsf=False, use_metamaterials=False,
                   point_source=(0, 0, 0), point_source_mask=0, steps=10, layout=0):
    size = _plane(size, mode, 1)
    names = ("x", "y", "z")

    def coord(v):
        v = _plane(v, mode, 0)
        return ",".join(f"{names[a]}:{v[a]}" for a in mode_axes(mode))

    args = [MODE_FLAGS[mode], "--size", coord(size),
            "--dx", repr(dx), "--wavelength", repr(wavelength), "--courant-factor", repr(courant),
            "--angle-teta", repr(teta), "--angle-phi", repr(phi), "--angle-psi", repr(psi),
            "--time-steps", str(steps), "--use-ca-cb", "--log-level", "0"]
    if layout:
        args += ["--layout-type", str(layout)]
    if use_pml:
        args += ["--use-pml", "--pml-size", coord(pml), "--use-ca-cb-pml"]
    if use_tfsf:
        args += ["--use-tfsf", "--tfsf-size-left", coord(tfsf_left), "--tfsf-size-right", coord(tfsf_right)]
    if use_metamaterials:
        args += ["--use-metamaterials"]
    if point_source_mask:
        args += ["--point-source", coord(point_source)]
        for k, name in enumerate(("ex", "ey", "ez", "hx", "hy", "hz")):
            if point_source_mask & (1 << k):
                args.append(f"--point-source-{name}")
    return args


def run_reference(materials=None, timeout=600, binary=None, extra_args=(), save=True, **kw):
    """Run the reference (the CPU build, or `binary` with `extra_args`, e.g.
    the CUDA build with --use-cuda); returns ({component: array}, the
    reference's own 'Total time' of the step loop in seconds).  save=False
    skips the field dumps (timing runs)."""
    binary = binary or REF_BIN
    if not os.path.exists(binary):
        raise FileNotFoundError(binary)
    mode = kw.get("mode", 3)
    size = _plane(kw.get("size", (20, 20, 20)), mode, 1)
    shape = tuple(size[a] for a in mode_axes(mode))
    with tempfile.TemporaryDirectory() as tmp:
        args = reference_args(**kw)
        flags = {"eps": "--load-eps-from-file", "mu": "--load-mu-from-file",
                 "omegape": "--load-omegape-from-file", "omegapm": "--load-omegapm-from-file",
                 "gammae": "--load-gammae-from-file", "gammam": "--load-gammam-from-file"}
        for name, arr in (materials or {}).items():
            p = os.path.join(tmp, f"{name}.txt")
            write_material_txt(p, np.asarray(arr).reshape(shape))
            args += [flags[name], p]
        names = ("x", "y", "z")
        end = ",".join(f"{names[a]}:{size[a]}" for a in mode_axes(mode))
        start = ",".join(f"{names[a]}:0" for a in mode_axes(mode))
        if save:
            args += ["--save-res", "--save-as-txt", "--manual-save-coords",
                     "--save-start-coord", start, "--save-end-coord", end]
        args += list(extra_args)
        r = subprocess.run([binary] + args, cwd=tmp, capture_output=True, text=True, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"reference failed ({r.returncode}): {r.stdout[-2000:]} {r.stderr[-2000:]}")
        total = None
        for line in r.stdout.splitlines():
            if line.startswith("Total time = "):
                total = float(line.split("=")[1].split()[0])
        out = {}
        for comp in COMPONENTS:
            files = glob.glob(os.path.join(tmp, f"previous-1_*_[[]name={comp}].txt"))
            if not files:
                continue
            data = np.loadtxt(files[0]).reshape(-1, len(shape) + 1)
            arr = np.zeros(shape)
            idx = tuple(data[:, i].astype(int) for i in range(len(shape)))
            arr[idx] = data[:, -1]
            out[comp] = arr
        return out, total
