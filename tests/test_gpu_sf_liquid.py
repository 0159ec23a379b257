"""Paracrystal and Percus-Yevick structure factors on the GPU against the golden fixtures made
by the reference's compiled liquid.cpp, and against the oracle on other grids and parameters.
Tolerance: FP64 kernels 1e-12 norm-wise; complex64 output 1e-6."""
import numpy as np
import pytest

import hipgisaxs_b200 as hg
from hipgisaxs_b200 import model

pytestmark = pytest.mark.gpu
LATT = {3: "cubic", 7: "hex"}


def _gpu(ctx, g, kind, a, out_type="c128"):
    if kind == "para":
        return model.sf_paracrystal(ctx, g, int(a[0]), LATT[int(a[1])], (a[2], a[3]), (a[4], a[5]),
                                    a[6], out_type=out_type)
    return model.sf_percus_yevick(ctx, g, a[0], a[1], int(a[2]), out_type=out_type)


@pytest.mark.parametrize("grid", ["g16", "g16abs"])
@pytest.mark.parametrize("case", ["para1d", "para2d_cubic", "para2d_hex", "py2d", "py3d"])
def test_golden_fixtures(ctx, po, golden, golden_grid, grid, case):
    d = golden(f"sfliq_{case}_{grid}")
    G, _ = golden_grid(grid)
    g = hg.QGrid.from_arrays(ctx, G.qx, G.qy, G.qz_ext)
    kind = str(d["kind"])
    assert po.rel_err(_gpu(ctx, g, kind, d["args"]), d["sf"]) < 1e-12
    assert po.rel_err(_gpu(ctx, g, kind, d["args"], "c64"), d["sf"]) < 1e-6


def test_larger_grid_and_parameters_against_oracle(ctx, po):
    G = po.Grid(64, 48, -2.0, 0.0, 2.0, 3.0, 0.2, 10.0, (6e-6, 4e-8))
    g = hg.QGrid.create(ctx, 64, 48, -2.0, 0.0, 2.0, 3.0, G.alpha_i, G.k0, (6e-6, 4e-8))
    for dims, latt in ((1, 3), (2, 3), (2, 7)):
        args = (dims, latt, 7.5, 9.0, 0.8, 1.1, 150.0)
        ref = po.sf_paracrystal(G, *args)
        got = model.sf_paracrystal(ctx, g, dims, LATT[latt], (7.5, 9.0), (0.8, 1.1), 150.0)
        assert po.rel_err(got, ref) < 1e-12
    for dims in (2, 3):
        for dia, vf in ((5.0, 0.1), (12.0, 0.45)):
            ref = po.sf_percus_yevick(G, dia, vf, dims)
            assert po.rel_err(model.sf_percus_yevick(ctx, g, dia, vf, dims), ref) < 1e-12


def test_percus_yevick_small_q_branch(ctx, po):
    """q-points at and near q = 0 (the reference's |q| < 1e-6 value) and at small q d, where
    the reference's PYFcn loses its value to cancellation (order-one terms cancelling to
    O((q d)^6)) and can return NaN.  The kernel reproduces the reference there: the same NaN
    positions, and elsewhere each value within 10x the oracle's own spread under 1e-15
    relative perturbations of q, plus 1e-12 of the value."""
    qx = np.array([0.0, 1e-7, 1e-5, 1e-3, 0.05, 0.3])
    qy = np.array([0.0, 2e-7, 0.0, 2e-3, 0.02, -0.4])
    qz = np.concatenate([np.zeros(6), np.full(6, 1e-4)]) + 0j
    g = hg.QGrid.from_arrays(ctx, qx, qy, qz)
    for dims in (2, 3):
        ref = po.sf_percus_yevick_arrays(9.0, 0.3, dims, qx, qy, qz)
        got = model.sf_percus_yevick(ctx, g, 9.0, 0.3, dims)
        nan = np.isnan(ref.real)
        np.testing.assert_array_equal(np.isnan(got.real), nan)
        spread = np.zeros(len(ref))
        for seed in range(4):
            r = np.random.default_rng(seed)
            alt = po.sf_percus_yevick_arrays(9.0, 0.3, dims, qx * (1 + 1e-15 * r.standard_normal(6)),
                                             qy * (1 + 1e-15 * r.standard_normal(6)), qz)
            spread = np.maximum(spread, np.nan_to_num(np.abs(alt - ref), nan=np.inf))
        ok = ~nan
        assert np.all(np.abs(got - ref)[ok] <= 10 * spread[ok] + 1e-12 * np.abs(ref[ok]))
        # away from q = 0 (q d >= 0.45 here) the values are well conditioned
        assert po.rel_err(got[4:6], ref[4:6]) < 1e-12


def test_invalid_selections_rejected(ctx, po):
    G = po.Grid(8, 6, -1.0, 0.0, 1.0, 2.0, 0.16, 10.0)
    g = hg.QGrid.from_arrays(ctx, G.qx, G.qy, G.qz_ext)
    with pytest.raises(hg.HgxError):
        model.sf_paracrystal(ctx, g, 2, "fcc", (1, 1), (0.1, 0.1), 10.0)
    with pytest.raises(hg.HgxError):
        model.sf_paracrystal(ctx, g, 3, "cubic", (1, 1), (0.1, 0.1), 10.0)
    with pytest.raises(hg.HgxError):
        model.sf_percus_yevick(ctx, g, 5.0, 0.2, 1)
