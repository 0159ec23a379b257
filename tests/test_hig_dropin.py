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
    r = subprocess.run([exe, hig], capture_output=True, text=True, timeout=300, cwd=str(tmp_path))
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
