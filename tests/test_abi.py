"""C-ABI checks that need no GPU: the library builds for sm_100a, loads,
exports every entry point include/fdtd_b200.h declares, and rejects bad
configurations before touching the device."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "fdtd_b200.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^[a-z_0-9 \*]*?\b(fdtd_[a-z_0-9]+) \(", text, re.M)))


def test_header_declares_entry_points():
    names = declared_functions()
    for n in ("fdtd_create", "fdtd_step", "fdtd_download_field", "fdtd_destroy", "fdtd_sync"):
        assert n in names


def test_library_exports_every_declared_symbol(fdtd):
    lib = fdtd.load_library()
    for name in declared_functions():
        assert hasattr(lib, name), name
    assert set(fdtd.EXPORTED) <= set(declared_functions())


def test_status_strings(fdtd):
    lib = fdtd.load_library()
    assert lib.fdtd_status_str(0) == b"ok"
    assert b"argument" in lib.fdtd_status_str(-1)


@pytest.mark.parametrize("bad", [
    dict(mode=9),
    dict(mode=1),
    dict(size=(2, 10, 10)),
    dict(use_pml=True, pml=10, size=(12, 12, 12)),
    dict(use_tfsf=True, tfsf_left=0, tfsf_right=3),
    dict(use_metamaterials=True),
    dict(dx=-1.0),
    dict(layout=2),
    dict(current_phase=3),
    dict(current_source_mask=1 << 6),
    dict(double_material_precision=True, use_metamaterials=True, use_pml=True, pml=2),
])
def test_create_rejects_bad_config(fdtd, bad):
    lib = fdtd.load_library()
    kw = dict(mode=3, size=(12, 12, 12))
    kw.update(bad)
    cfg = fdtd.make_config(**kw)
    h = ctypes.c_void_p()
    st = lib.fdtd_create(ctypes.byref(cfg), 0, ctypes.byref(h))
    assert st == -1
    assert not h.value
    assert lib.fdtd_last_error()


def test_create_without_gpu_fails_loudly(fdtd):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(fdtd.FdtdError):
        fdtd.Simulation(mode=3, size=(12, 12, 12))


def test_null_handles_are_rejected(fdtd):
    lib = fdtd.load_library()
    assert lib.fdtd_step(None, 0, 1) == -1
    assert lib.fdtd_sync(None, 0) == -1
    assert lib.fdtd_launch_count(None) == -1
    lib.fdtd_destroy(None)
