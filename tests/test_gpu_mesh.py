"""Triangle meshes on the GPU: the reference's triangle-parameter conversion, the DWBA chi^2
of a mesh, and its gradient with respect to every vertex coordinate (adjoint) against FP64
central differences of the oracle's chi^2.

Tolerances (norm-wise relative): intensity and chi^2 1e-5 (FP32C form factor); vertex
gradient 1e-4 of the FP64 finite-difference gradient (FP32 backward pass)."""
import numpy as np
import pytest

import hipgisaxs_b200 as hg
from hipgisaxs_b200 import fitting, meshes, model

pytestmark = pytest.mark.gpu
SUB = (4.88e-6, 7.37e-8, 0.0, -1)
DN2 = (-2 * 4.88e-6, -2 * 7.37e-8)


def test_mesh_conversion_matches_oracle(ctx, po):
    V, F = meshes.icosphere(8.0, 2, jitter=0.2)
    F = np.vstack([F, [[0, 0, 1]], [[3, 4, 3]]])  # two degenerate faces
    got = fitting.mesh_to_shape_def(ctx, V, F)
    ref = po.mesh_to_shape_def(V, F)  # drops the degenerate faces
    assert len(ref) == len(F) - 2
    np.testing.assert_allclose(got[:-2], ref, rtol=1e-13, atol=1e-13)
    assert np.all(got[-2:, 0] == 0.0)
    with pytest.raises(hg.HgxError):
        fitting.mesh_to_shape_def(ctx, V, np.array([[0, 1, len(V)]]))


def _oracle_chi2(po, G, fc, sd, R, counts, mask, scale, w=1.0):
    F = po.ff_approx_triangle(sd, G.qx, G.qy, G.qz_ext, R)
    I = po.dwba_combine(fc, np.ones_like(fc), complex(*DN2) * F, w)
    return po.chi2(I, counts, mask, scale), I


def test_mesh_chi2_and_vertex_gradient(ctx, po):
    G = po.Grid(40, 32, -2.0, 0.0, 2.0, 3.0, 0.2, 10.0)
    g = hg.QGrid.create(ctx, 40, 32, -2.0, 0.0, 2.0, 3.0, G.alpha_i, G.k0)
    rowfc = model.propagation_coeffs(ctx, g, [SUB], G.k0, G.alpha_i, 0, per_row=True)
    fc = po.propagation_coeffs(G, [SUB], 0)
    R = po.rot_mul(po.rot_axis(2, 0.3), po.rot_axis(0, 0.15))
    V, F = meshes.icosphere(8.0, 1, jitter=0.3, seed=5)
    Vt, _ = meshes.icosphere(8.5, 1, jitter=0.3, seed=6)
    rng = np.random.default_rng(8)
    _, It = _oracle_chi2(po, G, fc, po.mesh_to_shape_def(Vt, F), R, np.ones(G.n), None, 1.0)
    scale = 1e4 / It.max()
    counts = rng.poisson(scale * It).astype(float)
    mask = (rng.uniform(size=G.n) > 0.1).astype(np.uint32)

    chi, gv, inten = fitting.mesh_chi2_grad(ctx, g, V, F, rowfc, DN2, counts, mask, scale, 1.0, R,
                                            want_grad=True, want_intensity=True)
    sd = po.mesh_to_shape_def(V, F)
    ref_chi, ref_I = _oracle_chi2(po, G, fc, sd, R, counts, mask, scale)
    assert po.rel_err(inten, ref_I) < 1e-5
    assert abs(chi - ref_chi) < 1e-5 * ref_chi

    def chi_at(Vx):
        return _oracle_chi2(po, G, fc, po.mesh_to_shape_def(Vx, F), R, counts, mask, scale)[0]

    h = 1e-3
    fd = np.zeros_like(V)
    for i in range(len(V)):
        for k in range(3):
            def central(hh):
                Vp, Vm = V.copy(), V.copy()
                Vp[i, k] += hh
                Vm[i, k] -= hh
                return (chi_at(Vp) - chi_at(Vm)) / (2 * hh)
            fd[i, k] = (4 * central(h / 2) - central(h)) / 3
    err = np.linalg.norm(gv - fd) / np.linalg.norm(fd)
    assert err < 1e-4, err


def test_mesh_chi2_rejects_complex_grid(ctx, po):
    G = po.Grid(16, 12, -2.0, 0.0, 2.0, 3.0, 0.2, 10.0)
    g = hg.QGrid.create(ctx, 16, 12, -2.0, 0.0, 2.0, 3.0, G.alpha_i, G.k0, (6e-6, 4e-8))
    V, F = meshes.icosphere(8.0, 1)
    with pytest.raises(hg.HgxError):
        fitting.mesh_chi2_grad(ctx, g, V, F, np.zeros(4 * 12, complex), DN2, np.ones(G.n))


def test_offset_mesh_vertex_gradient_across_tiles(ctx, po):
    """A 320-face mesh (three triangle tiles, put in Morton order by the forward) 380 nm from
    the origin: chi^2 against the oracle, the adjoint gradient of 20 vertices against FP64
    central differences of the oracle's chi^2 (the gradient lands on the caller's vertex
    order), and the plain FP64 forward + adjoint against both."""
    G = po.Grid(40, 32, -2.0, 0.0, 2.0, 3.0, 0.2, 10.0)
    g = hg.QGrid.create(ctx, 40, 32, -2.0, 0.0, 2.0, 3.0, G.alpha_i, G.k0)
    rowfc = model.propagation_coeffs(ctx, g, [SUB], G.k0, G.alpha_i, 0, per_row=True)
    fc = po.propagation_coeffs(G, [SUB], 0)
    R = po.rot_mul(po.rot_axis(2, -0.5), po.rot_axis(1, 0.25))
    off = np.array([300.0, -200.0, 100.0])
    V, F = meshes.icosphere(8.0, 2, jitter=0.3, seed=15)
    Vt, _ = meshes.icosphere(8.4, 2, jitter=0.3, seed=16)
    V, Vt = V + off, Vt + off
    assert len(F) == 320
    rng = np.random.default_rng(18)
    _, It = _oracle_chi2(po, G, fc, po.mesh_to_shape_def(Vt, F), R, np.ones(G.n), None, 1.0)
    scale = 1e4 / It.max()
    counts = rng.poisson(scale * It).astype(float)

    chi, gv, inten = fitting.mesh_chi2_grad(ctx, g, V, F, rowfc, DN2, counts, None, scale, 1.0, R,
                                            want_grad=True, want_intensity=True)
    ref_chi, ref_I = _oracle_chi2(po, G, fc, po.mesh_to_shape_def(V, F), R, counts, None, scale)
    assert po.rel_err(inten, ref_I) < 1e-5
    assert abs(chi - ref_chi) < 1e-5 * ref_chi

    def chi_at(Vx):
        return _oracle_chi2(po, G, fc, po.mesh_to_shape_def(Vx, F), R, counts, None, scale)[0]

    h = 1e-3
    pick = rng.choice(len(V), 20, replace=False)
    fd = np.zeros((len(pick), 3))
    for a, i in enumerate(pick):
        for k in range(3):
            def central(hh):
                Vp, Vm = V.copy(), V.copy()
                Vp[i, k] += hh
                Vm[i, k] -= hh
                return (chi_at(Vp) - chi_at(Vm)) / (2 * hh)
            fd[a, k] = (4 * central(h / 2) - central(h)) / 3
    err = np.linalg.norm(gv[pick] - fd) / np.linalg.norm(fd)
    assert err < 1e-4, err
    chi64, gv64, _ = fitting.mesh_chi2_grad(ctx, g, V, F, rowfc, DN2, counts, None, scale, 1.0, R,
                                            want_grad=True, precision="f64")
    assert abs(chi64 - ref_chi) < 1e-11 * ref_chi
    assert np.linalg.norm(gv64[pick] - fd) / np.linalg.norm(fd) < 1e-6
    assert np.linalg.norm(gv - gv64) / np.linalg.norm(gv64) < 1e-5
