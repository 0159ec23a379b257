"""The C++ HiG front end (hig::HipGISAXSG, hig::HiGObjectiveFunctionG, include/hgx_hig.hpp):
the test driver compiles and links against libhgx.so (CPU); the fitting block's accessors
(hgx_hig_fit_reference, hgx_hig_fit_algorithm) read what the reader holds (CPU); on the GPU
the driver's simulation, post-processing and objective values agree with the oracle and with
the Python API over the same C ABI."""
import os
import subprocess

import numpy as np
import pytest

import hipgisaxs_b200 as hg
from conftest import ROOT
from hipgisaxs_b200.hig import METRICS, read_hig

SRC = os.path.join(ROOT, "tests", "cpp", "test_hig_sim.cpp")
LIBDIR = os.path.join(ROOT, "hipgisaxs_b200")
HIG = os.path.join(ROOT, "tests", "golden", "hig")


def _build(tmp_path):
    exe = str(tmp_path / "test_hig_sim")
    env = dict(os.environ)
    env.pop("CC", None)
    env.pop("CXX", None)
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-I" + os.path.join(ROOT, "include"), SRC,
                        "-L" + LIBDIR, "-lhgx", "-Wl,-rpath," + LIBDIR, "-o", exe],
                       capture_output=True, text=True, env=env)
    assert r.returncode == 0, r.stderr
    return exe


def test_hig_driver_compiles_and_links(tmp_path):
    assert os.path.exists(_build(tmp_path))


def test_fit_block_accessors():
    d = read_hig(os.path.join(HIG, "fit_objective.hig"))
    assert d.fit_reference() == {"path": "ref.out", "mask": "", "npar": 40, "nperp": 28}
    algs = d.fit_algorithms()
    assert len(algs) == 1
    assert algs[0]["name"] == "pso" and algs[0]["metric"] == METRICS["sqrt_unit_l2"]
    # the full grammar fixture: every referencedata and algorithm field, as the JSON holds it
    g = read_hig(os.path.join(HIG, "full_grammar.hig"))
    rd = g.data["referencedata"]
    ref = g.fit_reference()
    assert (ref["path"], ref["mask"]) == (rd["path"], rd["mask"]) == ("ref/data.out", "ref/mask.out")
    assert (ref["npar"], ref["nperp"]) == (64, 33)
    algs = g.fit_algorithms()
    assert [a["name"] for a in algs] == [a["name"] for a in g.algorithms] == ["pso", "pounders"]
    for a, j in zip(algs, g.algorithms):
        assert a["tolerance"] == j["tolerance"] and a["regularization"] == j["regularization"]
        assert a["metric"] == METRICS[j["distance_metric"]]
    # no referencedata block: refused
    p = read_hig(os.path.join(HIG, "paracrystal.hig"))
    with pytest.raises(hg.HgxError):
        p.fit_reference()
    assert p.fit_algorithms() == []


def _write_case(tmp_path, ref_img, mask):
    src = open(os.path.join(HIG, "fit_objective.hig")).read()
    src = src.replace('referencedata = { path = "ref.out",',
                      'referencedata = { path = "ref.out", mask = "mask.txt",')
    (tmp_path / "fit.hig").write_text(src)
    nrow, ncol = ref_img.shape
    with open(tmp_path / "ref.out", "w") as f:
        for row in ref_img:
            f.write(" ".join(repr(float(v)) for v in row) + "\n")
    (tmp_path / "mask.txt").write_text(" ".join(str(int(m)) for m in mask) + "\n")
    return str(tmp_path / "fit.hig")


@pytest.mark.gpu
def test_hig_driver_matches_oracle_and_api(ctx, po, tmp_path):
    exe = _build(tmp_path)
    d = read_hig(os.path.join(HIG, "fit_objective.hig"))
    nrow, ncol = d.image_size()
    d.fit_update([5.0, 25.0, 12.0])
    ref_img = po.compute_gisaxs(d.data, HIG)
    mask = np.ones(nrow * ncol, dtype=np.uint32)
    mask[::5] = 0
    hig = _write_case(tmp_path, ref_img, mask)
    # the FP64 kernels (HGX_PRECISION=f64) for parity with the oracle at 1e-11
    env = dict(os.environ, HGX_PRECISION="f64")
    r = subprocess.run([exe, hig], capture_output=True, text=True, timeout=300, cwd=str(tmp_path), env=env)
    assert r.returncode == 0, (r.returncode, r.stdout + r.stderr)

    def load(name):
        return np.fromfile(tmp_path / name)

    meta = (tmp_path / "meta.txt").read_text().split("\n")
    nr, nc, k0 = meta[0].split()
    assert (int(nr), int(nc)) == (nrow, ncol)
    assert float(k0) == pytest.approx(d.beam()[0], rel=1e-15)
    assert meta[1] == "throws"
    assert meta[2].split() == ["radius", "spacing", "twist"]
    assert [float(v) for v in meta[3].split()] == [3, 7, 18, 30, 0, 30]
    assert [float(v) for v in meta[5].split()] == [4, 22, 5]
    assert [float(v) for v in meta[6].split()] == [5, 24, 15]
    assert meta[8].split() == [str(ncol), str(nrow), str(nrow * ncol), "3"]

    # the simulation as read, and after update_params, against the oracle
    d0 = read_hig(hig)
    want0 = po.compute_gisaxs(d0.data, HIG)
    sim0 = load("sim0.bin").reshape(nrow, ncol)
    assert np.abs(sim0 - want0).max() / np.abs(want0).max() < 1e-11
    # the drop-in's default, FP32C: within 1e-5 of the oracle
    sub = tmp_path / "f32c"
    sub.mkdir()
    hig32 = _write_case(sub, ref_img, mask)
    env32 = {k: v for k, v in os.environ.items() if k != "HGX_PRECISION"}
    r = subprocess.run([exe, hig32], capture_output=True, text=True, timeout=300, cwd=str(sub), env=env32)
    assert r.returncode == 0, (r.returncode, r.stdout + r.stderr)
    sim0_32 = np.fromfile(sub / "sim0.bin").reshape(nrow, ncol)
    assert np.abs(sim0_32 - want0).max() / np.abs(want0).max() < 1e-5
    assert not np.array_equal(sim0_32, sim0)
    sim1 = load("sim1.bin").reshape(nrow, ncol)
    assert np.abs(sim1 - ref_img).max() / np.abs(ref_img).max() < 1e-11
    txt = np.loadtxt(tmp_path / "sim1.out")
    np.testing.assert_allclose(txt, sim1, rtol=1e-5)
    # post-processing of sim1 against the oracle
    nrm, ok = po.normalize(sim1.ravel())
    assert ok
    np.testing.assert_array_equal(load("norm.bin"), nrm)
    assert po.rel_err(load("smear.bin").reshape(nrow, ncol), po.smear_gaussian(sim1, 1.5)) < 1e-14

    # the objective: the same C ABI through Python on the same reference data and mask
    x = [4.2, 21.0, 3.0]
    dd = read_hig(hig)
    got0 = dd.objective(ctx, x, ref_img, mask, "sqrt_unit_l2", 0.0)
    np.testing.assert_array_equal(load("dist0.bin"), got0)
    got1 = dd.objective(ctx, x, ref_img, mask, "sqrt_unit_l2", 0.5)
    np.testing.assert_array_equal(load("dist1.bin"), got1)
    got2 = dd.objective(ctx, x, ref_img, mask, "sqrt_c_l2_residual", 0.5)
    np.testing.assert_array_equal(load("dist2.bin"), got2)
    # and against the oracle's composition
    dd.fit_update(x)
    img = po.compute_gisaxs(dd.data, HIG)
    want = po.fit_distance("sqrt_unit_l2", ref_img.ravel(), img.ravel(), mask)
    np.testing.assert_allclose(load("dist0.bin"), want, rtol=1e-10)
    # a reference simulated at the truth: zero distance there
    assert abs(load("dist3.bin")[0]) < 1e-20


_REGION = ('referencedata = { path = "ref.out", fitregion = { type = "qspace", '
           'regmin = [ -0.8 0.05 ], regmax = [ 0.6 0.9 ] },')


def _regrid_hig():
    src = open(os.path.join(HIG, "fit_objective.hig")).read()
    return src.replace('referencedata = { path = "ref.out",', _REGION)


def test_override_qregion(tmp_path):
    (tmp_path / "r.hig").write_text(_regrid_hig())
    d = read_hig(str(tmp_path / "r.hig"))
    assert d.image_size() == (28, 40)
    d.override_qregion(30, 20)
    assert d.image_size() == (20, 30)
    assert d.param_resolution() == [30, 20]
    assert d.param_output_minpoint() == (-0.8, 0.05) and d.param_output_maxpoint() == (0.6, 0.9)
    # no fit region: the reference's zeros
    e = read_hig(os.path.join(HIG, "fit_objective.hig"))
    e.override_qregion(10, 12)
    assert e.param_output_minpoint() == (0.0, 0.0) and e.param_output_maxpoint() == (0.0, 0.0)
    # refused: no referencedata block, an empty size, a pixel-space output region
    with pytest.raises(hg.HgxError):
        read_hig(os.path.join(HIG, "paracrystal.hig")).override_qregion(10, 10)
    with pytest.raises(hg.HgxError):
        d.override_qregion(0, 10)
    (tmp_path / "p.hig").write_text(_regrid_hig().replace('type = "qspace", minpoint', 'type = "pixels", minpoint'))
    p = read_hig(str(tmp_path / "p.hig"))
    assert p.param_output_type() == "pixels"
    with pytest.raises(hg.HgxError):
        p.override_qregion(10, 10)


@pytest.mark.gpu
def test_objective_regrids_to_reference(ctx, po, tmp_path):
    """A reference image of another size: the C++ objective re-grids the simulation over the
    fit region (override_qregion) and its values equal the Python API's after the same
    override, and the oracle's composition on the re-gridded description."""
    exe = _build(tmp_path)
    hig = tmp_path / "fit.hig"
    hig.write_text(_regrid_hig())
    d = read_hig(str(hig))
    d.override_qregion(30, 20)
    d.fit_update([5.0, 25.0, 12.0])
    ref_img = po.compute_gisaxs(d.data, HIG)
    assert ref_img.shape == (20, 30)
    with open(tmp_path / "ref.out", "w") as f:
        for row in ref_img:
            f.write(" ".join(repr(float(v)) for v in row) + "\n")
    r = subprocess.run([exe, str(hig), "regrid"], capture_output=True, text=True, timeout=300,
                       cwd=str(tmp_path))
    assert r.returncode == 0, (r.returncode, r.stdout + r.stderr)
    assert (tmp_path / "regrid.txt").read_text().split() == ["40", "28", "30", "20", "30", "20"]
    got = np.fromfile(tmp_path / "dist_regrid.bin")
    x = [4.2, 21.0, 3.0]
    e = read_hig(str(hig))
    e.override_qregion(30, 20)
    np.testing.assert_array_equal(got, e.objective(ctx, x, ref_img, None, "sqrt_unit_l2", 0.0))
    e.fit_update(x)
    img = po.compute_gisaxs(e.data, HIG)
    sim = e.compute_gisaxs(ctx)
    assert np.abs(sim - img).max() / np.abs(img).max() < 1e-11
    want = po.fit_distance("sqrt_unit_l2", ref_img.ravel(), img.ravel(), None)
    np.testing.assert_allclose(got, want, rtol=1e-10)


@pytest.mark.gpu
def test_run_all_gisaxs_writes_the_reference_files(ctx, po, tmp_path):
    """HipGISAXSG::run_all_gisaxs on a scan: one .out file per (alpha_i, phi, tilt) named as the
    reference names them, and the per-alpha_i sums, under runname_<timestamp>; their values are
    the Python API's images (which the GPU scan test holds against the oracle) at the .out
    text's 6 significant digits."""
    import ctypes
    import glob
    exe = _build(tmp_path)
    hig = os.path.join(HIG, "sim_scan.hig")
    r = subprocess.run([exe, hig, "scan"], capture_output=True, text=True, timeout=600, cwd=str(tmp_path))
    assert r.returncode == 0, (r.returncode, r.stdout + r.stderr)
    outdir = (tmp_path / "scan.txt").read_text().strip()
    assert os.path.basename(outdir).startswith("simscan_") and len(os.path.basename(outdir)) == len("simscan_") + 15
    files = sorted(os.path.basename(f) for f in glob.glob(os.path.join(tmp_path, outdir, "*.out")))
    d = read_hig(hig)
    ctypes.CDLL(None).srand(1)  # as the driver seeds it
    images, sums = d.run_all_gisaxs(ctx)

    def fmt(v):
        return "%g" % v

    want = {f"gisaxs_ai={fmt(a)}_rot={fmt(p)}_tilt={fmt(t)}.out": img for a, p, t, img in images}
    want.update({f"gisaxs_ai={fmt(a)}_averaged.out": img for a, img in sums.items()})
    assert files == sorted(want)
    for name, img in want.items():
        got = np.loadtxt(os.path.join(tmp_path, outdir, name))
        np.testing.assert_allclose(got, img, rtol=1e-5, atol=0)
