"""The C++ fitting front end (hig::HipGISAXSObjectiveFunctionG, include/hgx_hig.hpp): the test
driver compiles and links against libhgx.so (CPU); on the GPU its operator(),
value_and_gradient, batched evaluate and simulate agree with the Python batch API on the same
model, and its regularisation is the reference's (alpha/2)||x - x_mean||^2."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

SRC = os.path.join(ROOT, "tests", "cpp", "test_objective.cpp")
LIBDIR = os.path.join(ROOT, "hipgisaxs_b200")


def _build(tmp_path):
    exe = str(tmp_path / "test_objective")
    env = dict(os.environ)
    env.pop("CC", None)
    env.pop("CXX", None)
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-I" + os.path.join(ROOT, "include"), SRC,
                        "-L" + LIBDIR, "-lhgx", "-Wl,-rpath," + LIBDIR, "-o", exe],
                       capture_output=True, text=True, env=env)
    assert r.returncode == 0, r.stderr
    return exe


def test_objective_driver_compiles_and_links(tmp_path):
    assert os.path.exists(_build(tmp_path))


@pytest.mark.gpu
def test_objective_matches_batch_api(ctx, po, tmp_path):
    import hipgisaxs_b200 as hg
    from hipgisaxs_b200 import fitting, model

    exe = _build(tmp_path)
    nrow, ncol = 48, 64
    k0 = po.k0_from_kev(10.0)
    ai = 0.20 * np.pi / 180
    g = hg.QGrid.create(ctx, ncol, nrow, -2.0, 0.0, 2.0, 3.0, ai, k0)
    rowfc = model.propagation_coeffs(ctx, g, [(4.88e-6, 7.37e-8, 0.0, -1)], k0, ai, 0, per_row=True)
    abc, _ = model.lattice_vectors("hex")
    dn2 = (-2 * 4.88e-6, -2 * 7.37e-8)

    def mb(x):
        return fitting.model_block(x[0], x[1], x[2], x[3], 0.05, 11, (20, 20, 1), dn2, (0, 0, 0),
                                   1.0, smooth_sampling=True)

    truth = np.array([5.15, 9.6, 20.4, np.deg2rad(5.0)])
    fwd = fitting.CylinderBatch(ctx, g, rowfc, abc, [[0, 0, nrow, ncol]], precision="f64")
    target = fwd.forward([mb(truth)])[0].ravel()
    fwd.close()
    scale = 1e4 / target.max()
    counts = np.random.default_rng(3).poisson(scale * target).astype(np.float64)
    pop = np.array([[5.0, 10.0, 20.0, 0.0], [5.2, 9.7, 20.3, 0.05], [4.8, 10.4, 19.5, -0.1]])
    d = tmp_path
    np.array([nrow, ncol, scale], float).tofile(d / "meta.bin")
    counts.tofile(d / "counts.bin")
    pop.tofile(d / "x.bin")
    r = subprocess.run([exe, str(d)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    vg = np.fromfile(d / "value_grad.bin")
    op = np.fromfile(d / "op.bin")
    pp = np.fromfile(d / "pop.bin").reshape(-1, 5)
    img = np.fromfile(d / "image.bin")

    b = fitting.CylinderBatch(ctx, g, rowfc, abc, [[0, 0, nrow, ncol]] * len(pop),
                              np.tile(counts, len(pop)), None, scale, "f32c")
    chi, grad = b.eval([mb(x) for x in pop])
    # same kernels, same inputs: the C++ class and the batch API agree to rounding
    np.testing.assert_allclose(vg[0], chi[0], rtol=1e-12)
    np.testing.assert_allclose(vg[1:5], grad[0], rtol=1e-12, atol=1e-12 * np.abs(grad[0]).max())
    assert op[0] == vg[0]
    np.testing.assert_allclose(pp[:, 0], chi, rtol=1e-12)
    np.testing.assert_allclose(pp[:, 1:], grad, rtol=1e-12, atol=1e-12 * np.abs(grad).max())
    inten = b.forward([mb(pop[0])] + [mb(x) for x in pop[1:]])[0].ravel()
    np.testing.assert_allclose(img, inten, rtol=1e-12)
    # regularisation alpha = 2 about (5, 10, 20, 0)
    dx = pop[0] - np.array([5.0, 10.0, 20.0, 0.0])
    np.testing.assert_allclose(vg[5], vg[0] + 0.5 * 2.0 * dx @ dx, rtol=1e-12)
    np.testing.assert_allclose(vg[6:10], vg[1:5] + 2.0 * dx, rtol=1e-12, atol=1e-9)
    b.close()
    g.close()
