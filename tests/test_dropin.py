"""The C++ drop-in classes (include/hgx_hig.hpp): the test driver compiles and links against
libhgx.so (CPU); on the GPU it runs with the reference's signatures and its outputs match
the oracle."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, assert_exact_ff_close

SRC = os.path.join(ROOT, "tests", "cpp", "test_dropin.cpp")
LIBDIR = os.path.join(ROOT, "hipgisaxs_b200")


def _build(tmp_path):
    exe = str(tmp_path / "test_dropin")
    env = dict(os.environ)
    env.pop("CC", None)
    env.pop("CXX", None)
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-I" + os.path.join(ROOT, "include"), SRC,
                        "-L" + LIBDIR, "-lhgx", "-Wl,-rpath," + LIBDIR, "-o", exe],
                       capture_output=True, text=True, env=env)
    assert r.returncode == 0, r.stderr
    return exe


def test_dropin_compiles_and_links(tmp_path):
    assert os.path.exists(_build(tmp_path))


def test_dropin_compiles_inside_reference_tree():
    """hig_dropin.cpp against the reference's own class declarations (-DHGX_IN_REFERENCE_TREE),
    by the oracle Makefile's recipe; skipped where the reference sources are absent."""
    env = dict(os.environ)
    env.pop("CC", None)
    env.pop("CXX", None)
    ref = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "print-ref"],
                         capture_output=True, text=True, env=env).stdout.strip()
    if not ref or not os.path.isdir(os.path.join(ref, "include")):
        pytest.skip("reference sources not present")
    r = subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "dropin-check"],
                       capture_output=True, text=True, env=env)
    assert r.returncode == 0, r.stdout + r.stderr


@pytest.mark.gpu
def test_dropin_matches_oracle(ctx, po, tmp_path):
    exe = _build(tmp_path)
    G = po.Grid(24, 20, -2.0, 0.0, 2.0, 3.0, 0.2, 10.0)
    d = tmp_path
    np.array([G.nrow, G.ncol], float).tofile(d / "meta.bin")
    G.qx.tofile(d / "qx.bin")
    G.qy.tofile(d / "qy.bin")
    G.qz.tofile(d / "qz.bin")
    G.qz_ext.view(np.float64).tofile(d / "qz_ext.bin")
    rng = np.random.default_rng(1)
    T = 77
    sd = np.zeros((T, 8))
    sd[:, 0] = rng.uniform(0.2, 3.0, T)
    nrm = rng.normal(size=(T, 3))
    sd[:, 1:4] = nrm / np.linalg.norm(nrm, axis=1)[:, None]
    sd[:, 4:7] = rng.normal(scale=6.0, size=(T, 3))
    sd.tofile(d / "shape_def.bin")
    tris = rng.normal(scale=4.0, size=(23, 9))
    tris.tofile(d / "tris.bin")
    env = dict(os.environ, HGX_PRECISION="f64")
    r = subprocess.run([exe, str(d)], capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    rot = po.rot_mul(po.rot_axis(2, 0.3), po.rot_axis(0, 0.1))
    rd = lambda name: np.fromfile(d / name).view(np.complex128)
    assert po.rel_err(rd("out_ff_tri.bin"), po.ff_approx_triangle(sd, G.qx, G.qy, G.qz_ext, rot)) < 1e-12
    assert_exact_ff_close(po, rd("out_ff_exact.bin"), tris, G.qx, G.qy, G.qz_ext, rot)
    # the class receives explicit samples (radii 4.5, 5, 5.5; heights 9, 10), summed unweighted;
    # the oracle sums single-size cylinders (going through param_distribution would drop the
    # end values that its stepping lands on exactly)
    cyl = sum(po.ff_analytic_arrays("cylinder", [dict(type="radius", min=r, max=r),
                                                 dict(type="height", min=h, max=h)],
                                    G.qx, G.qy, G.qz_ext, 0.0, 0.0, (0.5, -1.0, 2.0), rot)
              for r in (4.5, 5.0, 5.5) for h in (9.0, 10.0))
    assert po.rel_err(rd("out_cyl.bin"), cyl) < 1e-12
    abc = np.array(po.lattice_vectors("hex")[:3])
    sf = po.sf_lattice(G, abc, [20, 20, 1], [20, 20, 20], (1, 2, 3), rot)
    assert po.rel_err(rd("out_sf.bin"), sf) < 1e-12
    # sphere: radii 9, 10 with weights 0.4, 0.6
    sph = 0.4 * po.ff_analytic_arrays("sphere", [dict(type="radius", min=9, max=9)], G.qx, G.qy,
                                      G.qz_ext, 0, 0, (0.5, -1.0, 2.0), rot) + \
        0.6 * po.ff_analytic_arrays("sphere", [dict(type="radius", min=10, max=10)], G.qx, G.qy,
                                    G.qz_ext, 0, 0, (0.5, -1.0, 2.0), rot)
    assert po.rel_err(rd("out_sph.bin"), sph) < 1e-12
    # the default (FP32-compensated) path through the same call
    r = subprocess.run([exe, str(d)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0
    assert po.rel_err(rd("out_ff_tri.bin"), po.ff_approx_triangle(sd, G.qx, G.qy, G.qz_ext, rot)) < 1e-5
