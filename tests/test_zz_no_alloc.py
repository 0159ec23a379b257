"""The allocation-free entry point, hgx_ff_triangles_noalloc.

It exists for callers that cannot allocate device memory: a plug-in living inside another
framework's memory pool that is handed only device pointers, a service held to a fixed
device-memory budget, or a real-time loop in which cudaMalloc would synchronise the device.
It keeps its scratch in a fixed static device array instead.  Here it is called through the
C ABI and checked against the allocating entry point (hgx_ff_triangles) on two calls in a
row with different meshes (so stale scratch from the first call cannot leak into the
second), within the FP32C tolerance used by the other tests (norm-wise 1e-5); after each
call its device error word must read 0, and the device's free memory must not change across
the second call.
"""
import numpy as np
import pytest

import hipgisaxs_b200 as hg
from hipgisaxs_b200 import _capi

pytestmark = pytest.mark.gpu
TOL32 = 1e-5


def _tri_cloud(rng, T, scale=6.0):
    sd = np.zeros((T, 8))
    sd[:, 0] = rng.uniform(0.2, 3.0, T)
    n = rng.normal(size=(T, 3))
    sd[:, 1:4] = n / np.linalg.norm(n, axis=1)[:, None]
    sd[:, 4:7] = rng.normal(scale=scale, size=(T, 3))
    return sd


def _noalloc(sd_d, qx_d, qy_d, qz_d, rot, out_d, stream):
    r = np.ascontiguousarray(rot, dtype=np.float64).reshape(9)
    return _capi.lib().hgx_ff_triangles_noalloc(
        sd_d.data_ptr(), sd_d.shape[0], qx_d.numel(), qx_d.data_ptr(), qy_d.data_ptr(),
        qz_d.numel(), qz_d.data_ptr(), r.ctypes.data, out_d.data_ptr(), _capi.C128, stream)


def _status(stream):
    import ctypes
    bits = ctypes.c_uint(0xFFFFFFFF)
    rc = _capi.lib().hgx_ff_triangles_noalloc_status(stream, ctypes.byref(bits))
    return rc, bits.value


def test_noalloc_matches_allocating_entry_on_two_calls(ctx, po):
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda:0")
    G = po.Grid(48, 40, -2.0, 0.0, 2.0, 3.0, 0.2, 10.0, (6e-6, 4e-8))
    rng = np.random.default_rng(2024)
    R1 = po.rot_mul(po.rot_axis(2, 0.3), po.rot_axis(0, 0.2))
    R2 = po.rot_axis(1, -0.4)
    qx_d = torch.tensor(G.qx, device=dev)
    qy_d = torch.tensor(G.qy, device=dev)
    qz_d = torch.tensor(G.qz_ext, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for call, (sd, R) in enumerate(((_tri_cloud(rng, 300), R1), (_tri_cloud(rng, 70), R2))):
        ref = hg.ff_triangles_arrays(ctx, sd, G.qx, G.qy, G.qz_ext, R, "f32c")
        out = torch.full((4 * G.n,), complex(np.nan, np.nan), dtype=torch.complex128, device=dev)
        sd_d = torch.tensor(sd, device=dev)
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info(dev)[0]
        _capi.check(_noalloc(sd_d, qx_d, qy_d, qz_d, R, out, stream))
        assert _status(stream) == (0, 0)
        torch.cuda.synchronize()
        if call == 1:  # the first call may load the library's device code; the second must not allocate
            assert torch.cuda.mem_get_info(dev)[0] == free0
        got = out.cpu().numpy()
        assert np.all(np.isfinite(got))
        assert po.rel_err(got, ref) < TOL32
        assert po.rel_err(got, po.ff_approx_triangle(sd, G.qx, G.qy, G.qz_ext, R)) < TOL32


def test_noalloc_rejects_sizes_beyond_its_fixed_scratch(ctx):
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda:0")
    sd_d = torch.zeros((65537, 8), dtype=torch.float64, device=dev)
    q_d = torch.zeros(4, dtype=torch.float64, device=dev)
    qz_d = torch.zeros(4, dtype=torch.complex128, device=dev)
    out = torch.zeros(4, dtype=torch.complex128, device=dev)
    rc = _noalloc(sd_d, q_d, q_d, qz_d, np.eye(3), out, 0)
    assert rc == 1
    assert b"65536" in _capi.lib().hgx_last_error()
