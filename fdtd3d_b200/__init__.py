"""fdtd3d_b200 - B200-native FDTD leapfrog step behind a C ABI.

The product is ``libfdtd_b200.so`` (built in-tree from ``csrc/`` by
``fdtd3d_b200.build``) exporting the functions declared in
``include/fdtd_b200.h``.  This module is a thin ctypes binding over that
library, used by the tests and ``bench.py``.  There is no CPU fallback: every
compute call goes to the CUDA library, and loading fails loudly when the
library is missing.
"""
from __future__ import annotations

import ctypes
import os
import struct

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfdtd_b200.so")

MODE_TMZ = 2
MODE_DIM3 = 3
MODE_TEX = 4
MODE_TEY = 5
MODE_TEZ = 6
MODE_TMX = 7
MODE_TMY = 8
MODE_EXHY = 10
MODE_EXHZ = 11
MODE_EYHX = 12
MODE_EYHZ = 13
MODE_EZHX = 14
MODE_EZHY = 15
# axes each mode keeps (its arrays are these axes, in x, y, z order, the last fastest)
KEPT_AXES = {MODE_DIM3: (0, 1, 2), MODE_TMZ: (0, 1), MODE_TEZ: (0, 1), MODE_TEX: (1, 2), MODE_TMX: (1, 2),
             MODE_TEY: (0, 2), MODE_TMY: (0, 2), MODE_EXHY: (2,), MODE_EYHX: (2,), MODE_EXHZ: (1,),
             MODE_EZHX: (1,), MODE_EYHZ: (0,), MODE_EZHY: (0,)}
PREC_FP64_PLAIN = 0
PREC_FP32 = 1
PREC_FP16S = 2
LAYOUT_E_CENTERED = 0   # --layout-type 0
LAYOUT_H_CENTERED = 1   # --layout-type 1
COMPONENTS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
MODE_COMPONENTS = {MODE_DIM3: COMPONENTS, MODE_TMZ: ("Ez", "Hx", "Hy"), MODE_TEZ: ("Ex", "Ey", "Hz"),
                   MODE_TEX: ("Ey", "Ez", "Hx"), MODE_TMX: ("Ex", "Hy", "Hz"), MODE_TEY: ("Ex", "Ez", "Hy"),
                   MODE_TMY: ("Ey", "Hx", "Hz"), MODE_EXHY: ("Ex", "Hy"), MODE_EXHZ: ("Ex", "Hz"),
                   MODE_EYHX: ("Ey", "Hx"), MODE_EYHZ: ("Ey", "Hz"), MODE_EZHX: ("Ez", "Hx"),
                   MODE_EZHY: ("Ez", "Hy")}
MATERIALS = ("eps", "mu", "omegape", "omegapm", "gammae", "gammam")
REDUCE_ENERGY = 0
REDUCE_L2 = 1

EXPORTED = (
    "fdtd_create", "fdtd_upload_material", "fdtd_upload_field", "fdtd_step", "fdtd_sync",
    "fdtd_download_field", "fdtd_upload_material_device", "fdtd_download_field_device",
    "fdtd_reduce", "fdtd_scalars", "fdtd_launch_count", "fdtd_destroy", "fdtd_status_str",
    "fdtd_last_error", "fdtd_stream", "fdtd_profile", "fdtd_kernel_time", "fdtd_step_kernel",
    "fdtd_batch_create", "fdtd_batch_upload_eps", "fdtd_batch_tune", "fdtd_batch_step", "fdtd_batch_sync",
    "fdtd_batch_download", "fdtd_batch_info", "fdtd_batch_last_error", "fdtd_batch_destroy",
    "fdtd_objective", "fdtd_backward", "fdtd_dft_setup", "fdtd_dft_read", "fdtd_ntff", "fdtd_keep_previous_level",
    "fdtd_upload_material_async", "fdtd_download_field_async", "fdtd_download_field_scattered",
    "fdtd_incident_length", "fdtd_download_incident", "fdtd_set_wait_limit", "fdtd_batch_set_wait_limit",
    "fdtd_inject_alloc_failure",
)


class FdtdError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str = ""):
        self.status = status
        super().__init__(f"{where}: status {status} ({detail})")


class Config(ctypes.Structure):
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
        ("point_source_kind", ctypes.c_int),
        ("point_source_bandwidth", ctypes.c_double),
        ("precision", ctypes.c_int),
        ("layout", ctypes.c_int),
        ("source_phase", ctypes.c_int),
        ("current_source", ctypes.c_int * 3),
        ("current_source_mask", ctypes.c_int),
        ("current_phase", ctypes.c_int),
        ("double_material_precision", ctypes.c_int),
        ("reserved", ctypes.c_int * 1),
    ]


class AdjointCfg(ctypes.Structure):
    _fields_ = [
        ("steps", ctypes.c_uint32),
        ("checkpoint_every", ctypes.c_uint32),
        ("probe_lo", ctypes.c_int * 2),
        ("probe_hi", ctypes.c_int * 2),
        ("precision", ctypes.c_int),
        ("reserved", ctypes.c_int * 3),
    ]


_lib = None


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Loads the CUDA library; raises if it is absent (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `python -m fdtd3d_b200.build`")
    lib = ctypes.CDLL(path)
    vp, i, d, u32, i64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_uint32, ctypes.c_int64
    sig = {
        "fdtd_create": ([ctypes.POINTER(Config), i, ctypes.POINTER(vp)], i),
        "fdtd_upload_material": ([vp, i, vp], i),
        "fdtd_upload_field": ([vp, i, vp], i),
        "fdtd_step": ([vp, u32, u32], i),
        "fdtd_sync": ([vp, i64], i),
        "fdtd_download_field": ([vp, i, vp], i),
        "fdtd_upload_material_device": ([vp, i, vp], i),
        "fdtd_download_field_device": ([vp, i, vp], i),
        "fdtd_reduce": ([vp, i, vp], i),
        "fdtd_scalars": ([vp, vp], i),
        "fdtd_launch_count": ([vp], i64),
        "fdtd_step_kernel": ([vp], ctypes.c_char_p),
        "fdtd_destroy": ([vp], None),
        "fdtd_status_str": ([i], ctypes.c_char_p),
        "fdtd_last_error": ([], ctypes.c_char_p),
        "fdtd_stream": ([vp], vp),
        "fdtd_profile": ([vp, i], i),
        "fdtd_kernel_time": ([vp, ctypes.POINTER(d), ctypes.POINTER(i64)], i),
        "fdtd_batch_create": ([ctypes.POINTER(Config), i, vp, i, ctypes.POINTER(vp)], i),
        "fdtd_batch_upload_eps": ([vp, i, vp], i),
        "fdtd_batch_tune": ([vp, i, vp], i),
        "fdtd_batch_step": ([vp, u32, u32], i),
        "fdtd_batch_sync": ([vp, i64], i),
        "fdtd_batch_download": ([vp, i, i, vp], i),
        "fdtd_batch_info": ([vp, ctypes.POINTER(i64), ctypes.POINTER(i), ctypes.POINTER(d)], i),
        "fdtd_batch_last_error": ([vp], ctypes.c_char_p),
        "fdtd_batch_destroy": ([vp], None),
        "fdtd_objective": ([vp, ctypes.POINTER(AdjointCfg), vp], i),
        "fdtd_dft_setup": ([vp, i, i, i, i, vp], i),
        "fdtd_dft_read": ([vp, vp], i),
        "fdtd_backward": ([vp, ctypes.POINTER(AdjointCfg), vp, vp], i),
        "fdtd_ntff": ([vp, vp, vp, vp, d, i, vp, vp], i),
        "fdtd_keep_previous_level": ([vp, i], i),
        "fdtd_upload_material_async": ([vp, i, vp], i),
        "fdtd_download_field_async": ([vp, i, vp], i),
        "fdtd_download_field_scattered": ([vp, i, vp], i),
        "fdtd_incident_length": ([vp], i),
        "fdtd_download_incident": ([vp, i, vp, i], i),
        "fdtd_set_wait_limit": ([vp, i64], i),
        "fdtd_batch_set_wait_limit": ([vp, i64], i),
        "fdtd_inject_alloc_failure": ([i64], i),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def inject_alloc_failure(after: int) -> None:
    """Host-side fault injection: the next ``after`` device / pinned allocations
    of the library succeed, later ones fail with FDTD_ERR_NOMEM; ``after`` < 0
    turns it off (fdtd_inject_alloc_failure)."""
    load_library().fdtd_inject_alloc_failure(int(after))


def f32(x: float) -> float:
    """Rounds like std::stof: the reference parses its float flags to float."""
    return struct.unpack("f", struct.pack("f", float(x)))[0]


def _triple(v, default, kept=(0, 1, 2)):
    """Per-axis triple for a mode that keeps axes `kept`: a sequence as long
    as `kept` gives those axes in x, y, z order; dropped axes get `default`."""
    if v is None:
        t = [default] * 3
    elif isinstance(v, (int, np.integer)):
        t = [int(v)] * 3
    else:
        v = [int(a) for a in v]
        if len(v) == len(kept) and len(kept) < 3:
            t = [default] * 3
            for a, val in zip(kept, v):
                t[a] = val
        else:
            t = v + [default] * (3 - len(v))
    return tuple(t[a] if a in kept else default for a in range(3))


def make_config(*, mode=MODE_DIM3, size=(20, 20, 20), pml=None, tfsf_left=None, tfsf_right=None,
                dx=0.0005, wavelength=0.02, courant=0.5, teta=90.0, phi=0.0, psi=90.0,
                use_pml=False, use_tfsf=False, use_metamaterials=False,
                point_source=(0, 0, 0), point_source_mask=0, point_source_kind=0, point_source_bandwidth=0.0,
                precision=PREC_FP64_PLAIN, source_phase=0, layout=LAYOUT_E_CENTERED,
                current_source=(0, 0, 0), current_source_mask=0, current_phase=0,
                double_material_precision=False) -> Config:
    c = Config()
    c.mode = mode
    kept = KEPT_AXES.get(mode, (0, 1, 2))
    c.size[:] = _triple(size, 1, kept)
    c.pml[:] = _triple(pml, 0, kept)
    c.tfsf_left[:] = _triple(tfsf_left, 0, kept)
    c.tfsf_right[:] = _triple(tfsf_right, 0, kept)
    c.dx, c.wavelength, c.courant = f32(dx), f32(wavelength), f32(courant)
    c.angle_teta, c.angle_phi, c.angle_psi = f32(teta), f32(phi), f32(psi)
    c.use_pml, c.use_tfsf, c.use_metamaterials = int(use_pml), int(use_tfsf), int(use_metamaterials)
    c.point_source[:] = _triple(point_source, 0, kept)
    c.point_source_mask = int(point_source_mask)
    c.point_source_kind = int(point_source_kind)
    c.point_source_bandwidth = float(point_source_bandwidth)
    c.precision = int(precision)
    c.layout = int(layout)
    c.source_phase = int(source_phase)
    c.current_source[:] = _triple(current_source, 0, kept)
    c.current_source_mask = int(current_source_mask)
    c.current_phase = int(current_phase)
    c.double_material_precision = int(bool(double_material_precision))
    return c


class Simulation:
    """One device-resident simulation (one fdtd_ctx); ``layout`` picks the
    reference's E_CENTERED (default) or H_CENTERED Yee layout.

    Arrays are x-major with z fastest (3-D) or (x, y) with y fastest (TMz),
    the reference's CudaGrid linear order.  ``step`` is asynchronous; reads
    synchronise.
    """

    def __init__(self, device: int = 0, materials=None, **cfg):
        self.lib = load_library()
        self.cfg = make_config(**cfg)
        self.mode = self.cfg.mode
        size = tuple(self.cfg.size)
        self.shape = tuple(size[a] for a in KEPT_AXES.get(self.mode, (0, 1, 2)))
        self.cells = int(np.prod(self.shape))
        # eps and mu on the doubled grid with double_material_precision
        self.material_shape = (tuple(2 * s for s in self.shape) if self.cfg.double_material_precision
                               else self.shape)
        h = ctypes.c_void_p()
        self._check(self.lib.fdtd_create(ctypes.byref(self.cfg), device, ctypes.byref(h)), "fdtd_create")
        self._h = h
        self.t = 0
        for name, arr in (materials or {}).items():
            self.set_material(name, arr)

    def _check(self, st: int, where: str) -> None:
        if st != 0:
            detail = (self.lib.fdtd_last_error() or b"").decode()
            raise FdtdError(st, where, detail or (self.lib.fdtd_status_str(st) or b"").decode())

    def set_material(self, name: str, arr) -> None:
        a = np.ascontiguousarray(arr, dtype=np.float64).reshape(-1)
        want = int(np.prod(self.material_shape)) if name in ("eps", "mu") else self.cells
        if a.size != want:
            raise ValueError("material array size does not match the grid")
        self._check(self.lib.fdtd_upload_material(self._h, MATERIALS.index(name), a.ctypes.data), "upload_material")

    def set_material_device(self, name: str, dev_ptr: int) -> None:
        self._check(self.lib.fdtd_upload_material_device(self._h, MATERIALS.index(name), dev_ptr),
                    "upload_material_device")

    def set_field(self, comp, arr) -> None:
        k = COMPONENTS.index(comp) if isinstance(comp, str) else comp
        a = np.ascontiguousarray(arr, dtype=np.float64).reshape(-1)
        self._check(self.lib.fdtd_upload_field(self._h, k, a.ctypes.data), "upload_field")

    def step(self, n: int, t_start: int | None = None) -> None:
        t0 = self.t if t_start is None else t_start
        self._check(self.lib.fdtd_step(self._h, t0, n), "fdtd_step")
        self.t = t0 + n

    def sync(self, timeout_ns: int = -1) -> None:
        self._check(self.lib.fdtd_sync(self._h, timeout_ns), "fdtd_sync")

    def field(self, comp, out: np.ndarray | None = None) -> np.ndarray:
        k = COMPONENTS.index(comp) if isinstance(comp, str) else comp
        if out is None:
            out = np.empty(self.cells, dtype=np.float64)
        self._check(self.lib.fdtd_download_field(self._h, k, out.ctypes.data), "download_field")
        return out.reshape(self.shape)

    def scattered_field(self, comp) -> np.ndarray:
        """The component minus the incident wave on the TF/SF box's cells."""
        k = COMPONENTS.index(comp) if isinstance(comp, str) else comp
        out = np.empty(self.cells, dtype=np.float64)
        self._check(self.lib.fdtd_download_field_scattered(self._h, k, out.ctypes.data), "download_field_scattered")
        return out.reshape(self.shape)

    def incident(self, family: str = "E") -> np.ndarray:
        """The current 1-D incident grid (EInc or HInc)."""
        n = self.lib.fdtd_incident_length(self._h)
        out = np.empty(n, dtype=np.float64)
        self._check(self.lib.fdtd_download_incident(self._h, 0 if family == "E" else 1, out.ctypes.data, n),
                    "download_incident")
        return out

    def field_device(self, comp, dev_ptr: int) -> None:
        k = COMPONENTS.index(comp) if isinstance(comp, str) else comp
        self._check(self.lib.fdtd_download_field_device(self._h, k, dev_ptr), "download_field_device")

    def reduce(self, what: int = REDUCE_ENERGY) -> np.ndarray:
        out = np.zeros(6, dtype=np.float64)
        self._check(self.lib.fdtd_reduce(self._h, what, out.ctypes.data), "fdtd_reduce")
        return out[:1] if what == REDUCE_ENERGY else out

    def scalars(self) -> dict:
        out = np.empty(3)
        self._check(self.lib.fdtd_scalars(self._h, out.ctypes.data), "fdtd_scalars")
        return {"dt": out[0], "frequency": out[1], "rel_phase_velocity": out[2]}

    def launch_count(self) -> int:
        return int(self.lib.fdtd_launch_count(self._h))

    def keep_previous_level(self, on: bool = True) -> None:
        """FP32 / FP16 storage: keep the previous H level after every step() call (for ntff)."""
        self._check(self.lib.fdtd_keep_previous_level(self._h, int(bool(on))), "keep_previous_level")

    def set_wait_limit(self, limit_ns: int) -> None:
        """Time limit of one grid-barrier wait of the adjoint kernel (<= 0: the default, 2 s)."""
        self._check(self.lib.fdtd_set_wait_limit(self._h, int(limit_ns)), "set_wait_limit")

    def _adjoint_cfg(self, steps, every, probe_lo, probe_hi, precision):
        c = AdjointCfg()
        c.steps = int(steps)
        c.checkpoint_every = int(every)
        c.probe_lo[:] = [int(v) for v in probe_lo]
        c.probe_hi[:] = [int(v) for v in probe_hi]
        c.precision = int(precision)
        return c

    def objective(self, steps, probe_lo, probe_hi, precision=PREC_FP32) -> float:
        """J = sum over t < steps of sum over the probe box of Ez_t^2 (2-D TMz, from t = 0)."""
        c = self._adjoint_cfg(steps, 1, probe_lo, probe_hi, precision)
        out = ctypes.c_double()
        self._check(self.lib.fdtd_objective(self._h, ctypes.byref(c), ctypes.byref(out)), "fdtd_objective")
        return out.value

    def backward(self, steps, every, probe_lo, probe_hi, precision=PREC_FP32):
        """(J, dJ/d eps on the (nx, ny) grid) by the checkpointed adjoint."""
        c = self._adjoint_cfg(steps, every, probe_lo, probe_hi, precision)
        out = ctypes.c_double()
        grad = np.empty(self.shape, dtype=np.float64)
        self._check(self.lib.fdtd_backward(self._h, ctypes.byref(c), ctypes.byref(out), grad.ctypes.data),
                    "fdtd_backward")
        return out.value, grad

    def dft_setup(self, comp, axis: int, index: int, freqs) -> None:
        """Starts a running DFT of `comp` on the plane x_axis = index at the given frequencies (Hz)."""
        k = COMPONENTS.index(comp) if isinstance(comp, str) else int(comp)
        f = np.ascontiguousarray(freqs, dtype=np.float64).reshape(-1)
        self._check(self.lib.fdtd_dft_setup(self._h, k, int(axis), int(index), int(f.size), f.ctypes.data),
                    "fdtd_dft_setup")
        n = list(self.cfg.size)
        self._dft_shape = (int(f.size),) + tuple(v for a, v in enumerate(n) if a != int(axis))

    def dft(self) -> np.ndarray:
        """Complex running DFT, shape (frequencies, plane axis a, plane axis b)."""
        out = np.empty(int(np.prod(self._dft_shape)) * 2)
        self._check(self.lib.fdtd_dft_read(self._h, out.ctypes.data), "fdtd_dft_read")
        return (out[0::2] + 1j * out[1::2]).reshape(self._dft_shape)

    @property
    def step_kernel(self) -> str:
        """Kernel that performed the last field update (see fdtd_step_kernel)."""
        return self.lib.fdtd_step_kernel(self._h).decode()

    @property
    def stream(self) -> int:
        """cudaStream_t of the context (as an integer), for CUDA events."""
        return int(self.lib.fdtd_stream(self._h) or 0)

    def profile(self, enable: bool = True) -> None:
        self._check(self.lib.fdtd_profile(self._h, int(enable)), "fdtd_profile")

    def kernel_time(self):
        """(summed field-kernel milliseconds, timed launches) since the last call."""
        ms = ctypes.c_double()
        n = ctypes.c_int64()
        self._check(self.lib.fdtd_kernel_time(self._h, ctypes.byref(ms), ctypes.byref(n)), "fdtd_kernel_time")
        return ms.value, n.value

    @property
    def handle(self) -> int:
        return self._h.value

    def close(self) -> None:
        if getattr(self, "_h", None):
            self.lib.fdtd_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many 2-D TMz simulations of different sizes advanced by one persistent
    kernel launch per ``step`` call (captured in a CUDA graph), FP32.

    ``sizes`` is a list of (nx, ny); every instance has its point source at
    its centre and shares the physics given as keyword arguments."""

    def __init__(self, sizes, device: int = 0, **cfg):
        self.lib = load_library()
        cfg.setdefault("mode", MODE_TMZ)
        cfg.setdefault("precision", PREC_FP32)
        cfg.setdefault("size", (3, 3))
        self.cfg = make_config(**cfg)
        self.sizes = [(int(a), int(b)) for a, b in sizes]
        arr = (ctypes.c_int * (2 * len(self.sizes)))(*[v for pair in self.sizes for v in pair])
        h = ctypes.c_void_p()
        st = self.lib.fdtd_batch_create(ctypes.byref(self.cfg), len(self.sizes), arr, device, ctypes.byref(h))
        if st != 0:
            raise FdtdError(st, "fdtd_batch_create", (self.lib.fdtd_status_str(st) or b"").decode())
        self._h = h
        self.t = 0

    def _check(self, st: int, where: str) -> None:
        if st != 0:
            raise FdtdError(st, where, (self.lib.fdtd_batch_last_error(self._h) or b"").decode())

    def set_eps(self, i: int, eps) -> None:
        a = np.ascontiguousarray(eps, dtype=np.float64).reshape(-1)
        assert a.size == self.sizes[i][0] * self.sizes[i][1]
        self._check(self.lib.fdtd_batch_upload_eps(self._h, i, a.ctypes.data), "batch_upload_eps")

    def tune(self, steps: int = 8):
        out = (ctypes.c_int * 3)()
        self._check(self.lib.fdtd_batch_tune(self._h, steps, out), "batch_tune")
        self.t = 0
        return tuple(out)

    def step(self, n: int, t_start: int | None = None) -> None:
        t0 = self.t if t_start is None else t_start
        self._check(self.lib.fdtd_batch_step(self._h, t0, n), "batch_step")
        self.t = t0 + n

    def sync(self, timeout_ns: int = -1) -> None:
        self._check(self.lib.fdtd_batch_sync(self._h, timeout_ns), "batch_sync")

    def field(self, i: int, comp) -> np.ndarray:
        k = COMPONENTS.index(comp) if isinstance(comp, str) else comp
        nx, ny = self.sizes[i]
        out = np.empty(nx * ny)
        self._check(self.lib.fdtd_batch_download(self._h, i, k, out.ctypes.data), "batch_download")
        return out.reshape(nx, ny)

    def set_wait_limit(self, limit_ns: int) -> None:
        """Time limit of one wait at the batch kernel's grid barrier (<= 0: the default, 5 s)."""
        self._check(self.lib.fdtd_batch_set_wait_limit(self._h, int(limit_ns)), "batch_set_wait_limit")

    def info(self) -> dict:
        cells = ctypes.c_int64()
        graph = ctypes.c_int()
        ms = ctypes.c_double()
        self._check(self.lib.fdtd_batch_info(self._h, ctypes.byref(cells), ctypes.byref(graph), ctypes.byref(ms)),
                    "batch_info")
        return {"cells": cells.value, "graph": bool(graph.value), "last_ms": ms.value}

    def close(self) -> None:
        if getattr(self, "_h", None):
            self.lib.fdtd_batch_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ntff(sim_re: "Simulation", sim_im: "Simulation", left, right, teta: float, phis) -> np.ndarray:
    """NTFF values of the complex field sim_re + i sim_im (the sine- and
    cosine-source runs of one form, 3-D; FP32 / FP16-storage runs call
    keep_previous_level before stepping) over the box with faces at
    left / right, at polar angle teta and each azimuth in phis (radians)."""
    lib = sim_re.lib
    lo = (ctypes.c_int * 3)(*[int(v) for v in left])
    hi = (ctypes.c_int * 3)(*[int(v) for v in right])
    ph = np.ascontiguousarray(phis, dtype=np.float64)
    out = np.empty(ph.size, dtype=np.float64)
    st = lib.fdtd_ntff(sim_re._h, sim_im._h, lo, hi, float(teta), int(ph.size), ph.ctypes.data, out.ctypes.data)
    sim_re._check(st, "fdtd_ntff")
    return out
