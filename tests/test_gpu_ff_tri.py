"""Numeric (mesh) form factor on the GPU against the CPU oracle.

Tolerances (norm-wise relative error ||x - ref||_2 / ||ref||_2 over all q-points):
  FP64 kernel : 1e-12
  FP32C kernel: 1e-5  (the bound the project promises; typical values are ~1e-7)
"""
import numpy as np
import pytest

import hipgisaxs_b200 as hg
from hipgisaxs_b200 import meshes

pytestmark = pytest.mark.gpu
TOL64 = 1e-12
TOL32 = 1e-5


def tri_cloud(rng, T, scale=6.0):
    sd = np.zeros((T, 8))
    sd[:, 0] = rng.uniform(0.2, 3.0, T)
    n = rng.normal(size=(T, 3))
    sd[:, 1:4] = n / np.linalg.norm(n, axis=1)[:, None]
    sd[:, 4:7] = rng.normal(scale=scale, size=(T, 3))
    return sd


@pytest.mark.parametrize("grid", ["g16", "g16abs"])
@pytest.mark.parametrize("rot", ["id", "r3"])
def test_golden_fixtures(ctx, po, golden, golden_grid, grid, rot):
    d = golden(f"fftri_{grid}_{rot}")
    G, _ = golden_grid(grid)
    g = hg.QGrid.from_arrays(ctx, G.qx, G.qy, G.qz_ext)
    assert g.mode == (1 if grid == "g16" else 2)
    assert g.ncol == G.ncol and g.nrow == G.nrow
    f64 = hg.ff_triangles(ctx, g, d["shape_def"], d["rot"], precision="f64")
    assert po.rel_err(f64, d["ff"]) < TOL64
    f32 = hg.ff_triangles(ctx, g, d["shape_def"], d["rot"], precision="f32c")
    assert po.rel_err(f32, d["ff"]) < TOL32


@pytest.mark.parametrize("ntri", [1, 63, 64, 65, 200])
@pytest.mark.parametrize("ppt", [1, 2, 4, -2, -4, -8])  # negative: packed FP32x2 kernel
def test_ragged_triangle_counts_and_launch_shapes(ctx, po, golden_grid, ntri, ppt):
    rng = np.random.default_rng(ntri)
    G, _ = golden_grid("g16")
    sd = tri_cloud(rng, ntri)
    R = po.rot_mul(po.rot_axis(2, 0.2), po.rot_axis(1, 0.1))
    ref = po.ff_approx_triangle(sd, G.qx, G.qy, G.qz_ext, R)
    g = hg.QGrid.from_arrays(ctx, G.qx, G.qy, G.qz_ext)
    f32 = hg.ff_triangles(ctx, g, sd, R, "f32c", pixels_per_thread=ppt)
    assert po.rel_err(f32, ref) < TOL32
    f64 = hg.ff_triangles(ctx, g, sd, R, "f64")
    assert po.rel_err(f64, ref) < TOL64


def test_points_mode_for_irregular_q(ctx, po):
    rng = np.random.default_rng(7)
    n = 777
    qx, qy = rng.uniform(-2, 2, n), rng.uniform(-2, 2, n)
    qz = rng.uniform(0, 3, 3 * n) + 1j * rng.uniform(0, 0.01, 3 * n)
    sd = tri_cloud(rng, 130)
    g = hg.QGrid.from_arrays(ctx, qx, qy, qz)
    assert g.mode == 0
    ref = po.ff_approx_triangle(sd, qx, qy, qz)
    assert po.rel_err(hg.ff_triangles(ctx, g, sd, None, "f32c"), ref) < TOL32
    assert po.rel_err(hg.ff_triangles(ctx, g, sd, None, "f64"), ref) < TOL64


def test_born_single_block_rows(ctx, po, golden_grid):
    G, _ = golden_grid("g16")
    rng = np.random.default_rng(11)
    sd = tri_cloud(rng, 99)
    qz = G.qz + 0j
    g = hg.QGrid.from_arrays(ctx, G.qx, G.qy, qz)
    assert g.mode == 2 and g.nrow == G.nrow
    ref = po.ff_approx_triangle(sd, G.qx, G.qy, qz)
    assert po.rel_err(hg.ff_triangles(ctx, g, sd, None, "f32c"), ref) < TOL32


def test_reference_shaped_call(ctx, po, golden_grid):
    G, _ = golden_grid("g16abs")
    sd = tri_cloud(np.random.default_rng(2), 70)
    ref = po.ff_approx_triangle(sd, G.qx, G.qy, G.qz_ext)
    out = hg.ff_triangles_arrays(ctx, sd, G.qx, G.qy, G.qz_ext, None, "f64")
    assert po.rel_err(out, ref) < TOL64
    out = hg.ff_triangles_arrays(ctx, sd, G.qx, G.qy, G.qz_ext, None, "f32c")
    assert po.rel_err(out, ref) < TOL32


@pytest.mark.parametrize("dn2", [(0.0, 0.0), (6e-6, 4e-8)])
def test_reference_shaped_call_rows_first(po, dn2):
    """From the second reference-shaped FP32C call with host arrays of the same sizes on, on a
    grid with detector rows of at least 64 q-points, the row kernel starts from a row table
    read on the host while a side stream copies the 4N qz values and checks them.  Results
    equal the device-grid path bit for bit, with a pageable and with a pinned (mapped, written
    directly by the kernel) output; a qz that is not constant along a row fails the check and is
    computed again from the full qz, equal to a fresh context's full path; the next regular grid
    is back on the fast path.  Real (paired) and absorbing (complex) qz blocks."""
    torch = pytest.importorskip("torch")
    G = po.Grid(128, 24, -2.0, 0.0, 2.0, 3.0, 0.2, 10.0, dn2)
    sd = tri_cloud(np.random.default_rng(9), 300)
    ctx = hg.Context(0)
    g = hg.QGrid.from_arrays(ctx, G.qx, G.qy, G.qz_ext)
    assert g.mode == (1 if dn2 == (0.0, 0.0) else 2) and g.ncol == 128
    want = hg.ff_triangles(ctx, g, sd, None, "f32c")
    first = hg.ff_triangles_arrays(ctx, sd, G.qx, G.qy, G.qz_ext, None, "f32c")
    second = hg.ff_triangles_arrays(ctx, sd, G.qx, G.qy, G.qz_ext, None, "f32c")
    pinned = torch.zeros(4 * G.n, dtype=torch.complex128).pin_memory()
    hg.ff_triangles_arrays(ctx, sd, G.qx, G.qy, G.qz_ext, None, "f32c", out=pinned)
    for got in (first, second, pinned.numpy()):
        assert np.array_equal(got, want)
    assert po.rel_err(second, po.ff_approx_triangle(sd, G.qx, G.qy, G.qz_ext)) < TOL32
    # one q-point of block 0 off its row's value, in the middle of row 3
    qz2 = G.qz_ext.copy()
    qz2[3 * G.ncol + G.ncol // 2] += 0.01
    fresh = hg.Context(0)
    full = hg.ff_triangles_arrays(fresh, sd, G.qx, G.qy, qz2, None, "f32c")
    again = hg.ff_triangles_arrays(ctx, sd, G.qx, G.qy, qz2, None, "f32c")
    assert np.array_equal(again, full)
    assert po.rel_err(again, po.ff_approx_triangle(sd, G.qx, G.qy, qz2)) < TOL32
    back = hg.ff_triangles_arrays(ctx, sd, G.qx, G.qy, G.qz_ext, None, "f32c")
    assert np.array_equal(back, want)
    # one block (Born): a grid of other sizes, then the same sizes again on the fast path
    qzb = G.qz + 0j
    gb = hg.QGrid.from_arrays(ctx, G.qx, G.qy, qzb)
    assert gb.mode == 2 and gb.ncol == 128
    want_b = hg.ff_triangles(ctx, gb, sd, None, "f32c")
    for _ in range(2):
        assert np.array_equal(hg.ff_triangles_arrays(ctx, sd, G.qx, G.qy, qzb, None, "f32c"), want_b)
    # scattered q-points (runs of equal qz shorter than 64): the full path, every call
    perm = np.random.default_rng(3).permutation(G.n)
    qx3, qy3 = G.qx[perm], G.qy[perm]
    qz3 = G.qz_ext.reshape(4, G.n)[:, perm].ravel()
    ref3 = po.ff_approx_triangle(sd, qx3, qy3, qz3)
    for _ in range(2):
        assert po.rel_err(hg.ff_triangles_arrays(ctx, sd, qx3, qy3, qz3, None, "f32c"), ref3) < TOL32
    fresh.close()
    ctx.close()


def test_device_qgrid_matches_oracle(ctx, po):
    for dn2 in ((0.0, 0.0), (6e-6, 4e-8)):
        G = po.Grid(40, 30, -2.0, 0.0, 2.0, 3.0, 0.2, 10.0, dn2)
        g = hg.QGrid.create(ctx, 40, 30, -2.0, 0.0, 2.0, 3.0, G.alpha_i, G.k0, dn2)
        r = g.read()
        for k in ("qx", "qy", "qz", "alpha"):
            np.testing.assert_allclose(r[k], getattr(G, k), rtol=1e-13, atol=1e-13)
        np.testing.assert_allclose(r["qz_ext"], G.qz_ext, rtol=1e-12, atol=1e-12)
        assert g.mode == (1 if dn2 == (0.0, 0.0) else 2)


def test_device_inputs_async(ctx, po, golden_grid):
    torch = pytest.importorskip("torch")
    G, _ = golden_grid("g16")
    sd = tri_cloud(np.random.default_rng(4), 150)
    ref = po.ff_approx_triangle(sd, G.qx, G.qy, G.qz_ext)
    dev = torch.device("cuda:0")
    qx = torch.tensor(G.qx, device=dev)
    qy = torch.tensor(G.qy, device=dev)
    qz = torch.tensor(G.qz_ext, device=dev)
    g = hg.QGrid.from_arrays(ctx, qx, qy, qz, ncol=G.ncol)
    assert g.mode == 1
    out = torch.zeros(4 * G.n, dtype=torch.complex64, device=dev)
    hg.ff_triangles(ctx, g, torch.tensor(sd, device=dev), None, "f32c", out=out, out_type="c64")
    ctx.synchronize()
    assert po.rel_err(out.cpu().numpy(), ref) < TOL32


def test_config0_icosphere_born(ctx, po):
    """256 x 256 Born numeric FF of the 1280-triangle icosphere (R = 10 nm)."""
    V, F = meshes.icosphere(10.0, 3)
    sd = meshes.shape_def_from_mesh(V, F)
    G = po.Grid(256, 256, -1.0, 0.0, 1.0, 2.0, 0.16, 10.0)
    qz = G.qz + 0j
    ref = po.ff_approx_triangle(sd, G.qx, G.qy, qz)
    g = hg.QGrid.from_arrays(ctx, G.qx, G.qy, qz)
    f32 = hg.ff_triangles(ctx, g, sd, None, "f32c")
    f64 = hg.ff_triangles(ctx, g, sd, None, "f64")
    assert po.rel_err(f64, ref) < TOL64
    assert po.rel_err(f32, ref) < TOL32
    assert po.rel_err(np.abs(f32) ** 2, np.abs(ref) ** 2) < TOL32


def test_config2_mesh_fp32_vs_fp64_and_oracle_sample(ctx, po):
    """50,000-triangle star mesh, DWBA, full triangle count on a 256 x 256 detector of the
    config-2 q-range; FP32C against the FP64 kernel everywhere and the oracle on a sample."""
    V, F = meshes.star_mesh()
    sd = meshes.shape_def_from_mesh(V, F)
    assert len(sd) == 50000
    G = po.Grid(256, 256, -2.0, 0.0, 2.0, 3.0, 0.2, 10.0)
    g = hg.QGrid.from_arrays(ctx, G.qx, G.qy, G.qz_ext)
    f32 = hg.ff_triangles(ctx, g, sd, None, "f32c")
    f64 = hg.ff_triangles(ctx, g, sd, None, "f64")
    assert po.rel_err(f32, f64) < TOL32
    idx = np.random.default_rng(0).choice(G.n, 48, replace=False)
    qz = G.qz_ext.reshape(4, -1)[:, idx].ravel()
    ref = po.ff_approx_triangle(sd, G.qx[idx], G.qy[idx], qz)
    got64 = f64.reshape(4, -1)[:, idx].ravel()
    assert po.rel_err(got64, ref) < TOL64


def test_linearity_in_triangles(ctx, po, golden_grid):
    G, _ = golden_grid("g16")
    sd = tri_cloud(np.random.default_rng(9), 300)
    g = hg.QGrid.from_arrays(ctx, G.qx, G.qy, G.qz_ext)
    full = hg.ff_triangles(ctx, g, sd, None, "f64")
    parts = hg.ff_triangles(ctx, g, sd[:137], None, "f64") + hg.ff_triangles(ctx, g, sd[137:], None, "f64")
    assert po.rel_err(parts, full) < 1e-13


def test_errors_are_reported(ctx):
    g = hg.QGrid.from_arrays(ctx, np.zeros(4), np.zeros(4), np.ones(4, complex))
    with pytest.raises(hg.HgxError):
        hg.ff_triangles(ctx, g, np.zeros((0, 8)), None, "f32c")


def test_launch_shape_autotuner(ctx, po, golden_grid):
    """The tuner times the candidate shapes, stores the fastest in the grid, and automatic
    calls afterwards give the result of that shape chosen by hand."""
    G, _ = golden_grid("g16")
    sd = tri_cloud(np.random.default_rng(12), 300)
    g = hg.QGrid.from_arrays(ctx, G.qx, G.qy, G.qz_ext)
    best, ms, times = hg.ff_tune(ctx, g, sd, None, "c128", reps=2)
    assert best in (4, 2, 1, -2, -4, -8) and set(times) == {4, 2, 1, -2, -4, -8}
    assert ms == times[best] == min(times.values())
    auto = hg.ff_triangles(ctx, g, sd, None, "f32c")
    hand = hg.ff_triangles(ctx, g, sd, None, "f32c", pixels_per_thread=best)
    assert np.array_equal(auto, hand)
    ref = po.ff_approx_triangle(sd, G.qx, G.qy, G.qz_ext)
    assert po.rel_err(auto, ref) < TOL32
    # per-q-point grids have one shape
    rng = np.random.default_rng(3)
    gp = hg.QGrid.from_arrays(ctx, rng.uniform(-2, 2, 50), rng.uniform(-2, 2, 50),
                              rng.uniform(0, 3, 150) + 0.01j)
    assert gp.mode == 0 and hg.ff_tune(ctx, gp, sd)[0] == 0


# A mesh about 1.3 um from the origin: the phases q.c reach ~2,600 rad on these grids, so an
# FP32 phase would lose ~1e-4 rad per term; the tiles' FP64 anchors keep the FP32C error at
# the level of a centred mesh.
OFFSET = np.array([1000.0, -700.0, 300.0])
# pointwise bound on q-points with |F|^2 >= 1e-6 of the largest |F|^2 (relative error of F)
PW_FLOOR = 1e-6
PW_TOL = 2e-5


def pointwise_err(a, ref, floor=PW_FLOOR):
    a, ref = np.asarray(a).ravel(), np.asarray(ref).ravel()
    p = np.abs(ref) ** 2
    m = p >= floor * p.max()
    return float(np.max(np.abs(a[m] - ref[m]) / np.abs(ref[m])))


def _offset_star(offset=OFFSET):
    V, F = meshes.star_mesh()
    return meshes.shape_def_from_mesh(V + offset, F)


@pytest.mark.parametrize("ppt", [4, -4])
def test_offset_mesh_rows_kernel_vs_oracle(ctx, po, ppt):
    sd = _offset_star()
    R = po.rot_mul(po.rot_axis(2, 0.7), po.rot_axis(0, 0.3))
    G = po.Grid(48, 40, -2.0, 0.0, 2.0, 3.0, 0.2, 10.0)
    ref = po.ff_approx_triangle(sd, G.qx, G.qy, G.qz_ext, R)
    g = hg.QGrid.from_arrays(ctx, G.qx, G.qy, G.qz_ext)
    assert g.mode == 1
    f32 = hg.ff_triangles(ctx, g, sd, R, "f32c", pixels_per_thread=ppt)
    assert po.rel_err(f32, ref) < TOL32
    assert pointwise_err(f32, ref) < PW_TOL
    f64 = hg.ff_triangles(ctx, g, sd, R, "f64")
    assert po.rel_err(f64, ref) < 1e-11


def test_offset_mesh_points_kernel_vs_oracle(ctx, po):
    rng = np.random.default_rng(21)
    n = 1500
    qx, qy = rng.uniform(-2, 2, n), rng.uniform(-2, 2, n)
    qz = rng.uniform(0, 3, 2 * n) + 1j * rng.uniform(0, 1e-3, 2 * n)
    sd = _offset_star()
    R = po.rot_mul(po.rot_axis(1, -0.4), po.rot_axis(2, 1.1))
    g = hg.QGrid.from_arrays(ctx, qx, qy, qz)
    assert g.mode == 0
    ref = po.ff_approx_triangle(sd, qx, qy, qz, R)
    f32 = hg.ff_triangles(ctx, g, sd, R, "f32c")
    assert po.rel_err(f32, ref) < TOL32
    assert pointwise_err(f32, ref) < PW_TOL


def test_translation_is_a_phase_at_full_size(ctx, po):
    """Size-independent property on a 256 x 256 DWBA grid with all 50,000 triangles: moving
    the mesh by t multiplies F by e^{i (Rq).t} (phase formed in FP64 on the host)."""
    V, F = meshes.star_mesh()
    sd0 = meshes.shape_def_from_mesh(V, F)
    sd1 = meshes.shape_def_from_mesh(V + OFFSET, F)
    R = po.rot_mul(po.rot_axis(2, 0.7), po.rot_axis(0, 0.3))
    G = po.Grid(256, 256, -2.0, 0.0, 2.0, 3.0, 0.2, 10.0)
    g = hg.QGrid.from_arrays(ctx, G.qx, G.qy, G.qz_ext)
    f0 = hg.ff_triangles(ctx, g, sd0, R, "f64").reshape(4, -1)
    f1 = hg.ff_triangles(ctx, g, sd1, R, "f32c").reshape(4, -1)
    qz = G.qz_ext.reshape(4, -1).real
    q = np.stack([np.broadcast_to(G.qx, qz.shape), np.broadcast_to(G.qy, qz.shape), qz], -1)
    ph = np.exp(1j * ((q @ np.asarray(R).T) @ OFFSET))
    expect = ph * f0
    assert po.rel_err(f1, expect) < TOL32
    assert pointwise_err(f1, expect) < PW_TOL


def test_headline_workload_fp32c_vs_fp64(ctx):
    """The benchmark's workload at full size: the 50,000-triangle star mesh on a 2048 x 2048
    DWBA grid built on the device (10 keV, alpha_i 0.20 deg).  FP32C against the plain FP64
    kernel: norm-wise 1e-5 (measured 2.8e-7); on the q-points with |F|^2 >= 1e-6 of the largest,
    99 % within 1e-5 of their own amplitude (measured 2.5e-6); and linearity over the triangles
    (the two halves' form factors add up to the whole's) within 1e-6 norm-wise."""
    torch = pytest.importorskip("torch")
    V, F = meshes.star_mesh()
    sd = torch.tensor(meshes.shape_def_from_mesh(V, F), device="cuda:0")
    assert sd.shape[0] == 50000
    k0 = 2 * np.pi / (1.23984 / 10.0)  # 10 keV, as the benchmark sets it
    g = hg.QGrid.create(ctx, 2048, 2048, -2.0, 0.0, 2.0, 3.0, 0.20 * np.pi / 180, k0)
    assert g.mode == 1
    n = 4 * 2048 * 2048
    f32 = torch.empty(n, dtype=torch.complex64, device="cuda:0")
    f64 = torch.empty(n, dtype=torch.complex128, device="cuda:0")
    hg.ff_triangles(ctx, g, sd, None, "f32c", out=f32, out_type="c64")
    hg.ff_triangles(ctx, g, sd, None, "f64", out=f64, out_type="c128")
    ctx.synchronize()
    d = f32.to(torch.complex128) - f64
    assert float(torch.linalg.vector_norm(d) / torch.linalg.vector_norm(f64)) < TOL32
    a = f64.abs()
    big = a * a >= PW_FLOOR * float((a * a).max())
    rel = (d.abs()[big] / a[big]).float()
    sample = rel[torch.randperm(rel.numel(), device=rel.device)[:1 << 20]]
    assert float(torch.quantile(sample, 0.99)) < TOL32
    del d, a, big, rel, f64
    h1 = torch.empty(n, dtype=torch.complex64, device="cuda:0")
    h2 = torch.empty(n, dtype=torch.complex64, device="cuda:0")
    hg.ff_triangles(ctx, g, sd[:25000], None, "f32c", out=h1, out_type="c64")
    hg.ff_triangles(ctx, g, sd[25000:], None, "f32c", out=h2, out_type="c64")
    ctx.synchronize()
    s = h1.to(torch.complex128) + h2.to(torch.complex128)
    w = f32.to(torch.complex128)
    assert float(torch.linalg.vector_norm(s - w) / torch.linalg.vector_norm(w)) < 1e-6
    g.close()
