"""Analytic form factors, lattice structure factor, Fresnel coefficients, DWBA combination
and distances on the GPU, against the golden fixtures (the reference's own CPU code) and the
oracle.  FP64 kernels: norm-wise relative error below 1e-12."""
import glob
import os

import numpy as np
import pytest

import hipgisaxs_b200 as hg
from hipgisaxs_b200 import model
from conftest import GOLDEN

pytestmark = pytest.mark.gpu
TOL64 = 1e-12


def _names(prefix):
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, prefix + "*.npz")))


def _grid(ctx, golden_grid, name):
    G, g = golden_grid(name)
    return G, g, hg.QGrid.from_arrays(ctx, G.qx, G.qy, G.qz_ext)


@pytest.mark.parametrize("name", _names("ffana_"))
def test_analytic_golden(ctx, po, golden, golden_grid, name):
    d = golden(name)
    G, _, g = _grid(ctx, golden_grid, str(d["grid"]))
    shape = name.split("_")[1]
    ff = model.ff_analytic_params(ctx, g, shape, d["params"], float(d["tau"]), float(d["eta"]),
                                  d["transvec"], d["rot"])
    assert po.rel_err(ff, d["ff"]) < TOL64
    f32 = model.ff_analytic_params(ctx, g, shape, d["params"], float(d["tau"]), float(d["eta"]),
                                   d["transvec"], d["rot"], out_type="c64")
    assert po.rel_err(f32, d["ff"]) < 1e-6


@pytest.mark.parametrize("name", _names("sf_"))
def test_sf_golden(ctx, po, golden, golden_grid, name):
    d = golden(name)
    G, _, g = _grid(ctx, golden_grid, str(d["grid"]))
    sf = model.sf_lattice(ctx, g, d["abc"], d["repet"], d["scaling"], d["center"], d["rot"])
    assert po.rel_err(sf, d["sf"]) < TOL64


@pytest.mark.parametrize("name", _names("fc_"))
def test_fresnel_golden(ctx, po, golden, golden_grid, name):
    d = golden(name)
    G, gq, g = _grid(ctx, golden_grid, str(d["grid"]))
    layers = [tuple(l[:3]) + (int(l[3]),) for l in d["layers"]]
    fc = model.propagation_coeffs(ctx, g, layers, G.k0, G.alpha_i, int(d["order"]), alpha=G.alpha)
    assert po.rel_err(fc, d["fc"]) < TOL64
    rows = model.propagation_coeffs(ctx, g, layers, G.k0, G.alpha_i, int(d["order"]),
                                    alpha=G.alpha, per_row=True)
    np.testing.assert_array_equal(rows.reshape(-1, 4)[:, 0], fc[:G.n][::G.ncol])


def test_fresnel_on_device_grid(ctx, po):
    G = po.Grid(64, 96, -2.0, 0.0, 2.0, 3.0, 0.2, 10.0)
    g = hg.QGrid.create(ctx, 64, 96, -2.0, 0.0, 2.0, 3.0, G.alpha_i, G.k0)
    layers = [(4.88e-6, 7.37e-8, 0.0, -1)]
    fc = model.propagation_coeffs(ctx, g, layers, G.k0, G.alpha_i, 0)
    assert po.rel_err(fc, po.propagation_coeffs(G, layers, 0)) < TOL64


@pytest.mark.parametrize("shape,params", [
    ("cylinder", "cfg1"),
    ("sphere", [dict(type="radius", stat="gaussian", min=8, max=12, mean=10, deviation=0.5, nvalues=9)]),
    ("pyramid", [dict(type="xsize", stat="uniform", min=9, max=11, nvalues=3),
                 dict(type="ysize", min=10, max=10), dict(type="height", min=3, max=3),
                 dict(type="baseangle", stat="uniform", min=55, max=65, nvalues=2)]),
])
def test_analytic_vs_oracle_larger_grid(ctx, po, shape, params):
    if params == "cfg1":
        params = po.cylinder_params(5.0, 10.0, 0.05, 11)
    G = po.Grid(80, 60, -2.0, 0.0, 2.0, 3.0, 0.2, 10.0)
    g = hg.QGrid.from_arrays(ctx, G.qx, G.qy, G.qz_ext)
    R = po.rot_axis(2, 0.087)
    ff = model.ff_analytic_params(ctx, g, shape, params, 0.0, 0.0, (0, 0, -1.0), R)
    ref = po.ff_analytic(G, shape, params, 0.0, 0.0, (0, 0, -1.0), R)
    assert po.rel_err(ff, ref) < TOL64


def test_analytic_rejects_unimplemented_shape(ctx, po):
    G = po.Grid(8, 8, -1.0, 0.0, 1.0, 2.0, 0.2, 10.0)
    g = hg.QGrid.from_arrays(ctx, G.qx, G.qy, G.qz_ext)
    with pytest.raises(hg.HgxError):
        model.ff_analytic(ctx, g, "cylinder", [([5.0], None)])  # height missing
    out = np.zeros(g.nqz, complex)
    # truncated cone (ShapeName 7): the reference reports it unimplemented (ff_ana_cone.cpp:47-49)
    rc = hg._capi.lib().hgx_ff_analytic_params(ctx.handle, g.handle, 7, 0, None, 0.0, 0.0, None,
                                               None, out.ctypes.data, 0)
    assert rc == 1


def test_dwba_combine_and_saxs(ctx, po):
    rng = np.random.default_rng(5)
    n = 5000
    ff = rng.normal(size=4 * n) + 1j * rng.normal(size=4 * n)
    sf = rng.normal(size=4 * n) + 1j * rng.normal(size=4 * n)
    fc = rng.normal(size=4 * n) + 1j * rng.normal(size=4 * n)
    base = rng.uniform(size=n)
    got = model.dwba_combine(ctx, fc, sf, ff, 0.7, base.copy())
    ref = po.dwba_combine(fc, sf, ff, 0.7, base.copy())
    assert po.rel_err(got, ref) < TOL64
    got32 = model.dwba_combine(ctx, fc, sf, ff.astype(np.complex64), 0.7, base.copy())
    assert po.rel_err(got32, ref) < 1e-6
    saxs = model.dwba_combine(ctx, None, sf[:n], ff[:n], 2.0)
    np.testing.assert_allclose(saxs, np.abs(2.0 * sf[:n] * ff[:n]) ** 2, rtol=1e-13)


def test_distances(ctx, po):
    rng = np.random.default_rng(6)
    n = 100003
    ref = rng.poisson(20, n).astype(float)
    data = rng.uniform(0, 40, n)
    mask = (rng.uniform(size=n) > 0.1).astype(np.uint32)
    assert abs(model.chi2(ctx, data, ref, mask, 1.3) - po.chi2(data, ref, mask, 1.3)) < \
        1e-12 * po.chi2(data, ref, mask, 1.3)
    assert abs(model.abs_diff_square(ctx, ref, data, mask) - po.abs_diff_square(ref, data, mask)) < \
        1e-12 * po.abs_diff_square(ref, data, mask)
    np.testing.assert_array_equal(model.residual_vector(ctx, ref, data, mask), mask * (ref - data))
    # deterministic: the same value twice, bit for bit
    assert model.chi2(ctx, data, ref, mask, 1.3) == model.chi2(ctx, data, ref, mask, 1.3)


@pytest.mark.parametrize("name", [n for n in _names("ffana_") if n.split("_")[1] in
                                  ("cylinder", "sphere", "box") and n.endswith("g16")])
def test_analytic_golden_f32c(ctx, po, golden, golden_grid, name):
    """The FP32C analytic form factor (cylinders, spheres, boxes on a grid with real qz)
    against the compiled reference's values: norm-wise relative error below 1e-5."""
    d = golden(name)
    G, _, g = _grid(ctx, golden_grid, str(d["grid"]))
    assert g.mode == 1
    ff = model.ff_analytic_params(ctx, g, name.split("_")[1], d["params"], float(d["tau"]),
                                  float(d["eta"]), d["transvec"], d["rot"], precision="f32c")
    assert po.rel_err(ff, d["ff"]) < 1e-5


@pytest.mark.parametrize("name", [n for n in _names("sf_") if n.endswith("g16")])
def test_sf_golden_f32c(ctx, po, golden, golden_grid, name):
    """The FP32C lattice structure factor (closed form, FP64 angles) against the compiled
    reference's principal-branch values on a grid with real qz: norm-wise 1e-5."""
    d = golden(name)
    G, _, g = _grid(ctx, golden_grid, str(d["grid"]))
    assert g.mode == 1
    sf = model.sf_lattice(ctx, g, d["abc"], d["repet"], d["scaling"], d["center"], d["rot"],
                          precision="f32c")
    assert po.rel_err(sf, d["sf"]) < 1e-5


@pytest.mark.parametrize("nh,step", [(11, 1.0), (12, 1.0), (11, 0.3), (7, None)])
def test_cylinder_f32c_height_sums_wide_qz(ctx, nh, step):
    """The FP32C cylinder's height sum: evenly stepped samples sum their exponentials in closed
    form (a Dirichlet ratio, with its sign for an odd/even count when qz d passes multiples of
    2 pi), the rest sample by sample.  On a real-qz grid reaching qz = 25 1/nm (qz d up to
    25 rad), against the FP64 kernel: norm-wise 1e-5, and 2e-5 pointwise on the points with
    |F| >= 1e-2 of the largest."""
    import math
    k0 = 2 * math.pi / (1.23984 / 10.0)
    g = hg.QGrid.create(ctx, 48, 160, -3.0, 0.0, 3.0, 25.0, 0.2 * math.pi / 180, k0)
    assert g.mode == 1
    if step is None:  # not evenly stepped: the per-sample sum
        h = np.array([5.0, 5.7, 7.1, 8.0, 9.9, 11.3, 12.0])
    else:
        h = 5.0 + step * np.arange(nh)
    r = np.linspace(3.0, 4.0, 5)
    dims = [(r, None), (np.zeros(0), None), (h, None)]
    f64 = model.ff_analytic(ctx, g, "cylinder", dims, precision="f64")
    f32 = model.ff_analytic(ctx, g, "cylinder", dims, precision="f32c")
    rel = np.linalg.norm(f32 - f64) / np.linalg.norm(f64)
    assert rel < 1e-5, rel
    big = np.abs(f64) >= 1e-2 * np.abs(f64).max()
    pw = np.abs(f32 - f64)[big] / np.abs(f64)[big]
    assert pw.max() < 2e-5, pw.max()
