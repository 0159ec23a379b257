"""Exact (polyhedral) triangle form factor on the GPU against the oracle and the golden
fixtures made by the reference's compiled compute_exact_triangle.

Tolerance: point by point, the reference formula's own conditioning (tests/conftest.py
assert_exact_ff_close: 10x the oracle's spread under 1e-15 relative perturbations of the
vertices and of q, plus 1e-12 of the rms), because the formula's edge and vertex terms cancel
severely at small |q|; complex64 output adds 1e-6 of the rms (the store's rounding)."""
import numpy as np
import pytest

import hipgisaxs_b200 as hg
from hipgisaxs_b200 import meshes

from conftest import assert_exact_ff_close

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("grid", ["g16", "g16abs"])
@pytest.mark.parametrize("rot", ["id", "r3"])
def test_golden_fixtures(ctx, po, golden, golden_grid, grid, rot):
    d = golden(f"ffexact_{grid}_{rot}")
    G, _ = golden_grid(grid)
    # the oracle is bit-identical to the compiled reference on these inputs
    np.testing.assert_array_equal(po.ff_exact_triangle(d["tris"], G.qx, G.qy, G.qz_ext, d["rot"]),
                                  d["ff"])
    g = hg.QGrid.from_arrays(ctx, G.qx, G.qy, G.qz_ext)
    f64 = hg.ff_exact_triangles(ctx, g, d["tris"], d["rot"])
    assert_exact_ff_close(po, f64, d["tris"], G.qx, G.qy, G.qz_ext, d["rot"])
    f32 = hg.ff_exact_triangles(ctx, g, d["tris"], d["rot"], out_type="c64")
    assert_exact_ff_close(po, f32, d["tris"], G.qx, G.qy, G.qz_ext, d["rot"], extra=1e-6)


@pytest.mark.parametrize("ntri", [1, 31, 32, 33, 100])
def test_ragged_counts_against_oracle(ctx, po, ntri):
    rng = np.random.default_rng(ntri)
    tris = rng.normal(scale=4.0, size=(ntri, 9))
    G = po.Grid(20, 14, -2.0, 0.0, 2.0, 3.0, 0.2, 10.0, (6e-6, 4e-8))
    R = po.rot_mul(po.rot_axis(2, 0.4), po.rot_axis(1, -0.3))
    g = hg.QGrid.from_arrays(ctx, G.qx, G.qy, G.qz_ext)
    assert_exact_ff_close(po, hg.ff_exact_triangles(ctx, g, tris, R), tris, G.qx, G.qy, G.qz_ext, R)


def test_degenerate_triangles_contribute_nothing(ctx, po):
    rng = np.random.default_rng(5)
    good = rng.normal(scale=4.0, size=(40, 9))
    bad = np.repeat(rng.normal(size=(3, 3)), 3, axis=0).reshape(3, 9)  # three repeated vertices
    tris = np.vstack([good[:20], bad, good[20:]])
    G = po.Grid(16, 12, -1.0, 0.0, 1.0, 2.0, 0.16, 10.0)
    g = hg.QGrid.from_arrays(ctx, G.qx, G.qy, G.qz_ext)
    out = hg.ff_exact_triangles(ctx, g, tris)
    assert np.all(np.isfinite(out))
    assert_exact_ff_close(po, out, good, G.qx, G.qy, G.qz_ext)


def test_reference_shaped_call_on_a_closed_mesh(ctx, po):
    V, F = meshes.icosphere(8.0, 3)
    tris = po.mesh_triangles(V, F)
    G = po.Grid(48, 36, -1.0, 0.0, 1.0, 2.0, 0.16, 10.0)
    out = np.zeros(len(G.qz_ext), dtype=np.complex128)
    hg._capi.check(hg.lib().hgx_ff_exact_triangles(
        ctx.handle, tris.ctypes.data, len(tris), len(G.qx), G.qx.ctypes.data, G.qy.ctypes.data,
        len(G.qz_ext), G.qz_ext.ctypes.data, None, out.ctypes.data))
    assert_exact_ff_close(po, out, tris, G.qx, G.qy, G.qz_ext)
