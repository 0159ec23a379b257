"""HiG-driven device set-up (hgx_hig_qgrid) against the oracle's QGrid::create."""
import os

import numpy as np
import pytest

from conftest import ROOT
from hipgisaxs_b200.hig import read_hig

HIG = os.path.join(ROOT, "tests", "golden", "hig")


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["paracrystal.hig", "percus_yevick.hig", "full_grammar.hig"])
def test_hig_qgrid_matches_oracle(ctx, po, name):
    d = read_hig(os.path.join(HIG, name))
    (ymin, zmin), (ymax, zmax) = d.param_output_minpoint(), d.param_output_maxpoint()
    ncol, nrow = d.param_resolution()
    value, unit = d.photon_energy()
    kev = value / 1000 if unit == "ev" else value
    for dn2 in ((0.0, 0.0), (6e-6, 4e-8)):
        G = po.Grid(ncol, nrow, ymin, zmin, ymax, zmax, d.scattering_alphai()[0], kev, dn2)
        g = d.qgrid(ctx, dn2)
        assert (g.ncol, g.nrow) == (ncol, nrow)
        r = g.read()
        for k in ("qx", "qy", "qz", "alpha"):
            np.testing.assert_allclose(r[k], getattr(G, k), rtol=1e-13, atol=1e-13)
        np.testing.assert_allclose(r["qz_ext"], G.qz_ext, rtol=1e-12, atol=1e-12)


SIM = ["sim_cylinders_hcp.hig", "sim_two_structures.hig", "paracrystal.hig", "percus_yevick.hig",
       "include_main.hig", "sim_scaling.hig", "sim_scaling_mixed.hig", "sim_repetition.hig",
       "sim_orientations.hig", "sim_shapes.hig"]


def _srand(seed):
    import ctypes
    ctypes.CDLL(None).srand(seed)


@pytest.mark.gpu
@pytest.mark.parametrize("name", SIM)
def test_compute_gisaxs_matches_oracle(ctx, po, name):
    """HipGISAXS::compute_gisaxs from a HiG file on the device against the oracle's
    composition of the same steps (FP64).  The rand()-drawn orientations are seeded alike."""
    path = os.path.join(HIG, name)
    d = read_hig(path)
    _srand(11)
    img = d.compute_gisaxs(ctx)
    _srand(11)
    ref = po.compute_gisaxs(d.data, HIG)
    assert img.shape == ref.shape == d.image_size()
    assert np.all(np.isfinite(img)) and ref.max() > 0
    err = np.abs(img - ref).max() / np.abs(ref).max()
    assert err < 1e-11, err


@pytest.mark.gpu
def test_compute_gisaxs_f32c_mesh(ctx, po):
    """The mesh form factors in compensated FP32: within the FP32C kernel's tolerance."""
    d = read_hig(os.path.join(HIG, "sim_two_structures.hig"))
    _srand(3)
    img = d.compute_gisaxs(ctx, precision="f32c")
    _srand(3)
    ref = po.compute_gisaxs(d.data, HIG)
    assert np.abs(img - ref).max() / np.abs(ref).max() < 2e-5


@pytest.mark.gpu
def test_compute_gisaxs_device_output(ctx, po):
    torch = pytest.importorskip("torch")
    d = read_hig(os.path.join(HIG, "paracrystal.hig"))
    nrow, ncol = d.image_size()
    out = torch.zeros(nrow * ncol, dtype=torch.float64, device="cuda:0")
    d.compute_gisaxs(ctx, out=out)
    ctx.synchronize()
    ref = po.compute_gisaxs(d.data, HIG)
    assert np.abs(out.cpu().numpy().reshape(nrow, ncol) - ref).max() / np.abs(ref).max() < 1e-11


@pytest.mark.gpu
@pytest.mark.parametrize("edit,words", [
    (("resolution = [ 48 32 ]", "resolution = [ 48 32 ], nslices = 3"), "nslices"),
    (('stat = "range"', 'stat = "bragg"'), "bragg orientations"),
    (("spacing = [ 150 150 0 ],", 'spacing = [ 150 150 0 ], distribution = "random",'), "distribution"),
    (("alphai = { min = 0.175 }", "alphai = { min = 0.1, max = 0.2, step = 0.05 }"), "alpha_i"),
    (('scaling = 24,', 'scaling = 24, lattice = { a = { mean = 2, stddev = 0.1, stat = "uniform" } },'),
     "scaling statistic"),
    (('repetition = [ 6 4 2 ]', 'repetitiondist = { xrepetition = { stat = "gaussian", min = 2, max = 5 } }'),
     "repetition statistic"),
])
def test_compute_gisaxs_refuses_unsupported(ctx, tmp_path, edit, words):
    from hipgisaxs_b200 import HgxError
    text = open(os.path.join(HIG, "sim_cylinders_hcp.hig")).read()
    assert edit[0] in text
    p = tmp_path / "edited.hig"
    p.write_text(text.replace(edit[0], edit[1], 1))
    d = read_hig(str(p))
    with pytest.raises(HgxError) as e:
        d.compute_gisaxs(ctx)
    assert words in str(e.value)
