"""The CPU oracle (plain-C restatement) against the golden fixtures generated from the
reference's own compiled CPU code (tests/golden/gen_golden.py)."""
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN

GRIDS = ["g16", "g16abs"]


def _names(prefix):
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, prefix + "*.npz")))


@pytest.mark.parametrize("grid", GRIDS)
def test_qgrid(golden_grid, grid):
    G, g = golden_grid(grid)
    for k in ("qx", "qy", "qz", "alpha"):
        np.testing.assert_array_equal(getattr(G, k), g[k], err_msg=k)
    np.testing.assert_array_equal(G.qz_ext, g["qz_ext"])


@pytest.mark.parametrize("name", _names("fftri_"))
def test_ff_triangles(po, golden, golden_grid, name):
    d = golden(name)
    G, _ = golden_grid(str(d["grid"]))
    ff = po.ff_approx_triangle(d["shape_def"], G.qx, G.qy, G.qz_ext, d["rot"], "port")
    np.testing.assert_allclose(ff, d["ff"], rtol=1e-13, atol=1e-13 * np.abs(d["ff"]).max())


@pytest.mark.parametrize("name", _names("ffexact_"))
def test_ff_exact_triangles(po, golden, golden_grid, name):
    d = golden(name)
    G, _ = golden_grid(str(d["grid"]))
    ff = po.ff_exact_triangle(d["tris"], G.qx, G.qy, G.qz_ext, d["rot"], "port")
    np.testing.assert_allclose(ff, d["ff"], rtol=1e-13, atol=1e-13 * np.abs(d["ff"]).max())


@pytest.mark.parametrize("name", _names("sfliq_"))
def test_sf_liquid(po, golden, golden_grid, name):
    d = golden(name)
    G, _ = golden_grid(str(d["grid"]))
    a = d["args"]
    if str(d["kind"]) == "para":
        sf = po.sf_paracrystal(G, int(a[0]), int(a[1]), *a[2:])
    else:
        sf = po.sf_percus_yevick(G, a[0], a[1], int(a[2]))
    np.testing.assert_array_equal(sf, d["sf"])


@pytest.mark.parametrize("name", _names("smear_"))
def test_smearing(po, golden, name):
    d = golden(name)
    np.testing.assert_array_equal(po.smear_gaussian(d["image"], float(d["sigma"])), d["smeared"])


@pytest.mark.parametrize("name", _names("ffana_"))
def test_ff_analytic(po, golden, golden_grid, name):
    d = golden(name)
    G, _ = golden_grid(str(d["grid"]))
    shape = name.split("_")[1]
    P = d["params"]
    params = []
    inv_p = {v: k for k, v in po.PARAM.items()}
    inv_s = {v: k for k, v in po.STAT.items()}
    for row in P:
        params.append(dict(type=inv_p[int(row[0])], stat=inv_s[int(row[1])], min=row[2],
                           max=row[3], mean=row[4], deviation=row[5], nvalues=int(row[6])))
    ff = po.ff_analytic(G, shape, params, float(d["tau"]), float(d["eta"]), d["transvec"], d["rot"])
    np.testing.assert_allclose(ff, d["ff"], rtol=1e-12, atol=1e-12 * np.abs(d["ff"]).max())


@pytest.mark.parametrize("name", _names("sf_"))
def test_sf_lattice(po, golden, golden_grid, name):
    d = golden(name)
    G, _ = golden_grid(str(d["grid"]))
    sf = po.sf_lattice(G, d["abc"], d["repet"], d["scaling"], d["center"], d["rot"])
    np.testing.assert_allclose(sf, d["sf"], rtol=1e-12, atol=1e-12 * np.abs(d["sf"]).max())


@pytest.mark.parametrize("name", _names("fc_"))
def test_propagation_coeffs(po, golden, golden_grid, name):
    d = golden(name)
    G, _ = golden_grid(str(d["grid"]))
    layers = [tuple(l[:3]) + (int(l[3]),) for l in d["layers"]]
    fc = po.propagation_coeffs(G, layers, int(d["order"]))
    np.testing.assert_allclose(fc, d["fc"], rtol=1e-13, atol=1e-15)


def test_lattice_table(po):
    a, b, c, t = po.lattice_vectors("hex")
    np.testing.assert_allclose(b, [0.5, np.sqrt(3) / 2, 0])
    for kind, hkl in (("cubic", "100"), ("cubic", "110"), ("bcc", "100"), ("bcc", "110"),
                      ("fcc", "100"), ("fcc", "111"), ("fco", "100"), ("hcp", "100")):
        po.lattice_vectors(kind, hkl)
    with pytest.raises(ValueError):
        po.lattice_vectors("cubic", "111")
