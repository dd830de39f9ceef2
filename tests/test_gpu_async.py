"""Asynchronous host copies (fdtd_upload_material_async,
fdtd_download_field_async): a pipelined loop of upload / steps / download
gives exactly the results of the synchronous calls, for the FP64 plain form
and the FP32 sweep, and every snapshot holds the field of its own time."""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _pinned(n):
    return torch.empty(n, dtype=torch.float64).pin_memory()


@pytest.mark.parametrize("prec", [0, 1], ids=["fp64", "fp32"])
def test_async_pipeline_matches_synchronous_calls(fdtd, prec):
    n = (48, 40, 52)
    kw = dict(mode=3, size=n, use_pml=True, pml=6, use_tfsf=True, tfsf_left=10, tfsf_right=10, teta=30, phi=45,
              psi=0, precision=prec)
    rng = np.random.default_rng(3)
    eps_list = [np.where(rng.random(n) < 0.2, 4.0, 1.0) for _ in range(3)]
    cells = int(np.prod(n))
    # synchronous reference
    want = []
    with fdtd.Simulation(**kw) as sim:
        for eps in eps_list:
            sim.set_material("eps", eps)
            sim.step(7)
            want.append(sim.field("Ez").copy())
    # pipelined: uploads and downloads overlap the steps
    hosts_in = [_pinned(cells) for _ in eps_list]
    for h, eps in zip(hosts_in, eps_list):
        h.copy_(torch.from_numpy(eps.reshape(-1)))
    hosts_out = [_pinned(cells) for _ in eps_list]
    with fdtd.Simulation(**kw) as sim:
        lib = sim.lib
        for h_in, h_out in zip(hosts_in, hosts_out):
            sim._check(lib.fdtd_upload_material_async(sim._h, 0, ctypes.c_void_p(h_in.data_ptr())), "up")
            sim.step(7)
            sim._check(lib.fdtd_download_field_async(sim._h, 2, ctypes.c_void_p(h_out.data_ptr())), "down")
        sim.sync()
    for w, h in zip(want, hosts_out):
        got = h.numpy().reshape(w.shape)
        assert np.array_equal(got.view(np.int64), w.view(np.int64))
    assert not np.array_equal(want[0], want[1])
