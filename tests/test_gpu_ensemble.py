"""The grain loop of one structure on the device (hgx_dwba_mesh_grains) against the oracle's
composition of the reference's functions, grain by grain: the rotated numeric form factor,
the lattice structure factor at the grain's centre and rotation, the Fresnel coefficients and
the DWBA combination.  Tolerances (norm-wise relative): FP64 form factor 1e-12; FP32C 1e-5."""
import numpy as np
import pytest

import hipgisaxs_b200 as hg
from hipgisaxs_b200 import meshes, model

pytestmark = pytest.mark.gpu
SUB = (4.88e-6, 7.37e-8, 0.0, -1)


def _case(po):
    rng = np.random.default_rng(7)
    V, F = meshes.icosphere(4.0, 2)
    sd = meshes.shape_def_from_mesh(V, F)
    G = po.Grid(40, 30, -2.0, 0.0, 2.0, 3.0, 0.2, 10.0)
    ng = 5
    rots = [po.rot_mul(po.rot_mul(po.rot_axis(2, a), po.rot_axis(0, b)), po.rot_axis(1, c))
            for a, b, c in rng.uniform(-0.4, 0.4, (ng, 3))]
    centers = rng.normal(scale=3.0, size=(ng, 3))
    weights = rng.uniform(0.5, 1.5, ng)
    abc = np.array(po.lattice_vectors("hex")[:3])
    repet, scaling = (6.0, 6.0, 1.0), (14.0, 14.0, 14.0)
    dn2 = (-2 * 4.88e-6, -2 * 7.37e-8)
    fc = po.propagation_coeffs(G, [SUB], 0)
    ref = np.zeros(G.n)
    for R, c, w in zip(rots, centers, weights):
        ff = po.ff_approx_triangle(sd, G.qx, G.qy, G.qz_ext, R)
        sf = po.sf_lattice(G, abc, repet, scaling, c, R)
        ref = po.dwba_combine(fc, sf, complex(*dn2) * ff, w, ref)
    return G, sd, rots, centers, weights, abc, repet, scaling, fc, dn2, ref


@pytest.mark.parametrize("precision,tol", [("f64", 1e-12), ("f32c", 1e-5)])
def test_grain_loop_matches_oracle(ctx, po, precision, tol):
    G, sd, rots, centers, weights, abc, repet, scaling, fc, dn2, ref = _case(po)
    g = hg.QGrid.create(ctx, G.ncol, G.nrow, -2.0, 0.0, 2.0, 3.0, G.alpha_i, G.k0)
    got = model.dwba_mesh_grains(ctx, g, sd, rots, centers, weights, abc, repet, scaling, fc, dn2,
                                 precision)
    assert po.rel_err(got, ref) < tol


def test_grains_add_up(ctx, po):
    """Linearity over grains: the sum of the grain loop over two halves equals the whole."""
    G, sd, rots, centers, weights, abc, repet, scaling, fc, dn2, _ = _case(po)
    g = hg.QGrid.create(ctx, G.ncol, G.nrow, -2.0, 0.0, 2.0, 3.0, G.alpha_i, G.k0)
    args = (abc, repet, scaling, fc, dn2, "f64")
    whole = model.dwba_mesh_grains(ctx, g, sd, rots, centers, weights, *args)
    a = model.dwba_mesh_grains(ctx, g, sd, rots[:2], centers[:2], weights[:2], *args)
    b = model.dwba_mesh_grains(ctx, g, sd, rots[2:], centers[2:], weights[2:], *args)
    assert po.rel_err(a + b, whole) < 1e-13


def test_needs_a_dwba_grid(ctx, po):
    G, sd, rots, centers, weights, abc, repet, scaling, fc, dn2, _ = _case(po)
    gb = hg.QGrid.from_arrays(ctx, G.qx, G.qy, G.qz + 0j)  # Born: one qz block
    with pytest.raises(hg.HgxError):
        model.dwba_mesh_grains(ctx, gb, sd, rots, centers, weights, abc, repet, scaling, fc, dn2)


def test_structure_sum(ctx, po):
    rng = np.random.default_rng(8)
    I = rng.random((3, 20, 24))
    for r in ([0.2, 0.3, 0.5], [1.0, 2.0, 5.0]):      # summing to 1, and rescaled
        got = model.structure_sum(ctx, I, r)
        ref = po.structure_sum(I, r).reshape(20, 24)
        np.testing.assert_array_equal(got, ref)


def test_analytic_grain_loop_matches_oracle(ctx, po):
    """Cylinders on a hex lattice with five grain orientations (the config-1 model with a
    grain distribution) against the oracle's per-grain composition."""
    rng = np.random.default_rng(9)
    G = po.Grid(40, 30, -2.0, 0.0, 2.0, 3.0, 0.2, 10.0)
    ng = 5
    rots = [po.rot_axis(2, a) for a in rng.uniform(-0.5, 0.5, ng)]
    centers = rng.normal(scale=2.0, size=(ng, 3))
    weights = rng.uniform(0.5, 1.5, ng)
    abc = np.array(po.lattice_vectors("hex")[:3])
    params = po.cylinder_params(5.0, 10.0, 0.05, 5)
    tv = (0.5, -1.0, 0.0)
    dn2 = (-2 * 4.88e-6, -2 * 7.37e-8)
    fc = po.propagation_coeffs(G, [SUB], 0)
    ref = np.zeros(G.n)
    for R, c, w in zip(rots, centers, weights):
        ff = po.ff_analytic(G, "cylinder", params, 0.0, 0.0, tv, R)
        sf = po.sf_lattice(G, abc, (20, 20, 1), (20, 20, 20), c, R)
        ref = po.dwba_combine(fc, sf, complex(*dn2) * ff, w, ref)
    g = hg.QGrid.create(ctx, G.ncol, G.nrow, -2.0, 0.0, 2.0, 3.0, G.alpha_i, G.k0)
    got = model.dwba_analytic_grains(ctx, g, "cylinder", params, rots, centers, weights, abc,
                                     (20, 20, 1), (20, 20, 20), fc, dn2, transvec=tv)
    assert po.rel_err(got, ref) < 1e-12
