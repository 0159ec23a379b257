"""The fused cylinder-lattice model (configs 1, 3, 4): forward intensity against the oracle's
composition of the reference's functions (cylinder form factor, hex lattice structure factor,
Parratt coefficients, DWBA combination), chi^2, the adjoint gradient against central finite
differences and against FP64, and the batched graph-captured launch against single calls.

Tolerances (norm-wise relative): FP64 forward 1e-12; FP32C forward/chi^2/gradient 1e-5 of the
FP64 values; adjoint vs central differences (h = 1e-5 relative) 1e-6."""
import numpy as np
import pytest

import hipgisaxs_b200 as hg
from hipgisaxs_b200 import fitting, model

pytestmark = pytest.mark.gpu
SUB = (4.88e-6, 7.37e-8)
DN2 = (-2 * 4.88e-6, -2 * 7.37e-8)  # vacuum layer minus a Si-like particle


def _setup(ctx, po, ncol=96, nrow=64):
    G = po.Grid(ncol, nrow, -2.0, 0.0, 2.0, 3.0, 0.20, 10.0)
    g = hg.QGrid.create(ctx, ncol, nrow, -2.0, 0.0, 2.0, 3.0, G.alpha_i, G.k0)
    rowfc = model.propagation_coeffs(ctx, g, [(SUB[0], SUB[1], 0.0, -1)], G.k0, G.alpha_i, 0,
                                     per_row=True)
    abc, _ = model.lattice_vectors("hex")
    return G, g, rowfc, abc


def _oracle_intensity(po, G, m):
    R, H, a, phi, s, n = m[0], m[1], m[2], m[3], m[4], int(m[5])
    params = po.cylinder_params(R, H, s, n) if s > 0 else po.cylinder_params(R, H)
    rot = po.rot_axis(2, phi)
    ff = po.ff_analytic(G, "cylinder", params, 0.0, 0.0, (0, 0, 0), rot)
    dn2 = complex(m[9], m[10])
    abc = np.array(po.lattice_vectors("hex")[:3])
    sf = po.sf_lattice(G, abc, m[6:9], [a, a, a], m[11:14], rot)
    fc = po.propagation_coeffs(G, [(SUB[0], SUB[1], 0.0, -1)], 0)
    return po.dwba_combine(fc, sf, dn2 * ff, m[14])


def _model(R=5.0, H=10.0, a=20.0, phi=np.deg2rad(5.0), spread=0.05, n=11):
    return fitting.model_block(R, H, a, phi, spread, n, (20, 20, 1), DN2, (0, 0, 0), 1.0)


def test_forward_matches_oracle(ctx, po):
    G, g, rowfc, abc = _setup(ctx, po)
    m = _model()
    ref = _oracle_intensity(po, G, m)
    full = [0, 0, G.nrow, G.ncol]
    for prec, tol in (("f64", 1e-12), ("f32c", 1e-5)):
        b = fitting.CylinderBatch(ctx, g, rowfc, abc, [full], precision=prec)
        got = b.forward([m])[0].ravel()
        assert po.rel_err(got, ref) < tol, prec
        b.close()
    b = fitting.CylinderBatch(ctx, g, rowfc, abc, [full])
    assert po.rel_err(b.plain_forward(0, m), ref) < 1e-12


def test_forward_single_size_and_roi(ctx, po):
    G, g, rowfc, abc = _setup(ctx, po)
    m = _model(R=4.0, H=7.0, a=17.0, phi=0.3, spread=0.0, n=1)
    m[11:14] = (1.0, -2.0, 0.5)
    ref = _oracle_intensity(po, G, m).reshape(G.nrow, G.ncol)
    roi = [10, 20, 30, 50]
    b = fitting.CylinderBatch(ctx, g, rowfc, abc, [roi], precision="f64")
    got = b.forward([m])[0]
    assert po.rel_err(got, ref[10:40, 20:70]) < 1e-12


def _counts(ref, rng, peak=1e4):
    s = peak / ref.max()
    return rng.poisson(s * ref).astype(float), s


def test_chi2_and_adjoint_gradient(ctx, po):
    G, g, rowfc, abc = _setup(ctx, po)
    rng = np.random.default_rng(3)
    truth = _model(R=5.15, H=9.6, a=20.4, phi=np.deg2rad(5.0))
    counts, s = _counts(_oracle_intensity(po, G, truth), rng)
    m = _model()
    full = [0, 0, G.nrow, G.ncol]
    b64 = fitting.CylinderBatch(ctx, g, rowfc, abc, [full], counts, None, s, "f64")
    b32 = fitting.CylinderBatch(ctx, g, rowfc, abc, [full], counts, None, s, "f32c")
    c64, g64 = b64.eval([m])
    c32, g32 = b32.eval([m])
    ref_chi2 = po.chi2(_oracle_intensity(po, G, m), counts, None, s)
    assert abs(c64[0] - ref_chi2) < 1e-11 * ref_chi2
    assert abs(c32[0] - c64[0]) < 1e-5 * c64[0]
    assert np.linalg.norm(g32 - g64) < 1e-5 * np.linalg.norm(g64)
    # central differences of the FP64 chi^2.  The reference's param_distribution stepping
    # can change the number of size samples between R - h and R + h (R = 5: 10 samples,
    # R - 1e-5 R: 11), a jump, so differences are taken in the smooth sampling mode.
    m[15] = 1.0
    c64, g64 = b64.eval([m])
    c32, g32 = b32.eval([m])
    assert np.linalg.norm(g32 - g64) < 1e-5 * np.linalg.norm(g64)
    def central(j, h):
        mp, mm = m.copy(), m.copy()
        mp[j] += h
        mm[j] -= h
        return (b64.eval([mp])[0][0] - b64.eval([mm])[0][0]) / (2 * h)

    # Richardson-extrapolated central differences (h = 1e-5 relative, O(h^4) error): chi^2
    # varies sharply with phi and a through the 20-repetition lattice peaks
    fd = np.zeros(4)
    for j in range(4):
        h = 1e-5 * (abs(m[j]) if j < 3 else 1.0)
        fd[j] = (4 * central(j, h / 2) - central(j, h)) / 3
    np.testing.assert_allclose(g64[0], fd, rtol=1e-6, atol=1e-6 * np.abs(fd).max())


def test_batch_matches_single_calls_and_replays(ctx, po):
    G, g, rowfc, abc = _setup(ctx, po, 128, 96)
    rng = np.random.default_rng(11)
    counts_full, s = _counts(_oracle_intensity(po, G, _model()), rng)
    counts_full = counts_full.reshape(G.nrow, G.ncol)
    rois = [[0, 0, 96, 128], [5, 7, 40, 33], [50, 60, 46, 68], [10, 100, 17, 28], [0, 0, 1, 1]]
    counts = np.concatenate([counts_full[r0:r0 + nr, c0:c0 + nc].ravel() for r0, c0, nr, nc in rois])
    models = [_model(5 * (1 + 0.02 * i), 10 * (1 - 0.03 * i), 20 + 0.3 * i, 0.05 * i) for i in range(5)]
    batch = fitting.CylinderBatch(ctx, g, rowfc, abc, rois, counts, None, s, "f32c")
    chi, grad = batch.eval(models)
    for i, r in enumerate(rois):
        one = fitting.CylinderBatch(ctx, g, rowfc, abc, [r],
                                    counts[batch.offsets[i]:batch.offsets[i + 1]], None, s, "f32c")
        c1, g1 = one.eval([models[i]])
        assert c1[0] == chi[i] and np.array_equal(g1[0], grad[i])
        one.close()
    # graph replay with new parameters equals a fresh batch
    models2 = [m.copy() for m in models]
    for m in models2:
        m[0] *= 1.01
    chi2b, grad2b = batch.eval(models2)
    fresh = fitting.CylinderBatch(ctx, g, rowfc, abc, rois, counts, None, s, "f32c")
    c3, g3 = fresh.eval(models2)
    assert np.array_equal(chi2b, c3) and np.array_equal(grad2b, g3)


def test_batch_rejects_bad_input(ctx, po):
    G, g, rowfc, abc = _setup(ctx, po, 32, 24)
    with pytest.raises(hg.HgxError):
        fitting.CylinderBatch(ctx, g, rowfc, abc, [[0, 0, 25, 32]])  # ROI beyond the grid
    gabs = hg.QGrid.create(ctx, 32, 24, -2.0, 0.0, 2.0, 3.0, G.alpha_i, G.k0, (6e-6, 4e-8))
    with pytest.raises(hg.HgxError):
        fitting.CylinderBatch(ctx, gabs, rowfc, abc, [[0, 0, 24, 32]])  # complex qz
    fcc = np.array([[0, 0.5, 0.5], [0.5, 0, 0.5], [0.5, 0.5, 0]])
    with pytest.raises(hg.HgxError):  # lattice vectors out of the plane
        fitting.CylinderBatch(ctx, g, rowfc, fcc, [[0, 0, 24, 32]]).forward([_model()])


def test_tile_shapes_and_autotuner(ctx, po):
    """Every tile shape gives the same intensities (bit-identical: per-pixel work does not
    depend on the shape) and the same chi^2/gradient up to summation order; the tuner
    returns a shape of the table, and evaluations after it match that shape set by hand."""
    G, g, rowfc, abc = _setup(ctx, po, 128, 96)
    rng = np.random.default_rng(5)
    counts_full, s = _counts(_oracle_intensity(po, G, _model()), rng)
    counts_full = counts_full.reshape(G.nrow, G.ncol)
    rois = [[0, 0, 96, 128], [3, 9, 37, 61], [20, 30, 11, 5]]
    counts = np.concatenate([counts_full[r0:r0 + nr, c0:c0 + nc].ravel() for r0, c0, nr, nc in rois])
    models = [_model(5 * (1 + 0.02 * i), 10, 20 + 0.2 * i, 0.03 * i) for i in range(3)]
    shapes = fitting.CylinderBatch.shapes()
    assert len(shapes) >= 2 and all(t % 32 == 0 and p >= 1 for t, p in shapes)
    batch = fitting.CylinderBatch(ctx, g, rowfc, abc, rois, counts, None, s, "f64")
    assert batch.shape == 0
    chi0, grad0 = batch.eval(models)
    inten0 = batch.forward(models)
    for k, (t, p) in enumerate(shapes):
        batch.shape = k
        assert batch.shape == k
        assert batch.nitems == sum(-(-r[2] * r[3] // (t * p)) for r in rois)
        for a, b in zip(batch.forward(models), inten0):
            assert np.array_equal(a, b)
        chi, grad = batch.eval(models)
        np.testing.assert_allclose(chi, chi0, rtol=1e-12)
        assert po.rel_err(grad, grad0) < 1e-12
    best, ms, times = batch.tune(models, reps=2)
    assert 0 <= best < len(shapes) and batch.shape == best
    assert np.all(times > 0) and ms == times[best] == times.min()
    chi_t, grad_t = batch.eval(models)
    batch.shape = best
    chi_s, grad_s = batch.eval(models)
    assert np.array_equal(chi_t, chi_s) and np.array_equal(grad_t, grad_s)
    with pytest.raises(hg.HgxError):
        batch.shape = len(shapes)
