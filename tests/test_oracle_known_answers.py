"""Analytic known answers that pin the oracle independently of the reference code."""
import numpy as np
import pytest


def test_sf_at_q_zero_is_product_of_repetitions(po):
    abc = np.array(po.lattice_vectors("hex")[:3])
    z = np.zeros(3)
    sf = po.sf_lattice_arrays(abc, [20, 20, 1], [20, 20, 20], [0, 0, 0], None, z, z,
                              np.zeros(3, complex))
    np.testing.assert_allclose(sf, 400.0, rtol=1e-14)
    sf = po.sf_lattice_arrays(abc, [5, 7, 3], [20, 20, 20], [0, 0, 0], None, z, z,
                              np.zeros(3, complex))
    np.testing.assert_allclose(sf, 105.0, rtol=1e-14)


@pytest.mark.parametrize("k", [1, 2, 5])
def test_dirichlet_kernel_at_bragg_peaks(po, k):
    # a-axis only: q.a = 2 pi k gives |S_a| = N
    a = 20.0
    qx = np.array([2 * np.pi * k / a])
    abc = np.eye(3)
    sf = po.sf_lattice_arrays(abc, [10, 1, 1], [a, a, a], [0, 0, 0], None, qx, np.zeros(1),
                              np.zeros(1, complex))
    assert abs(abs(sf[0]) - 10.0) < 1e-6


def test_dirichlet_kernel_general(po):
    a, N = 20.0, 7
    qx = np.linspace(0.013, 1.9, 57)
    sf = po.sf_lattice_arrays(np.eye(3), [N, 1, 1], [a, a, a], [0, 0, 0], None, qx,
                              np.zeros_like(qx), np.zeros(len(qx), complex))
    th = qx * a
    ref = np.abs(np.sin(N * th / 2) / np.sin(th / 2))
    np.testing.assert_allclose(np.abs(sf), ref, rtol=1e-9)


def test_single_interface_parratt_is_fresnel(po):
    k0 = po.k0_from_kev(10.0)
    delta, beta = 4.88e-6, 7.37e-8
    stack = [(0j, 0.0), (complex(2 * delta, 2 * beta), 0.0)]
    ac = np.sqrt(2 * delta)
    for alpha in np.linspace(0.2 * ac, 5 * ac, 23):
        T, R = po.parratt(stack, alpha, k0, 0)
        kz0 = -k0 * np.sqrt(np.sin(alpha) ** 2 + 0j)
        kz1 = -k0 * np.sqrt(np.sin(alpha) ** 2 - complex(2 * delta, 2 * beta))
        r = (kz0 - kz1) / (kz0 + kz1)
        assert abs(T - 1) < 1e-14
        assert abs(R - r) < 1e-12 * max(1, abs(r))
        if alpha < 0.8 * ac:
            assert abs(R) > 0.9  # total external reflection below the critical angle


def test_rotation_moves_into_triangles(po):
    rng = np.random.default_rng(3)
    T = 40
    sd = np.zeros((T, 8))
    sd[:, 0] = rng.uniform(0.5, 2, T)
    n = rng.normal(size=(T, 3))
    sd[:, 1:4] = n / np.linalg.norm(n, axis=1)[:, None]
    sd[:, 4:7] = rng.normal(scale=5, size=(T, 3))
    R = po.rot_mul(po.rot_axis(2, 0.4), po.rot_axis(0, -0.3))
    qx, qy = rng.uniform(-1, 1, 30), rng.uniform(-1, 1, 30)
    qz = rng.uniform(0, 2, 30) + 0j
    f1 = po.ff_approx_triangle(sd, qx, qy, qz, R)
    sd2 = sd.copy()
    sd2[:, 1:4] = sd[:, 1:4] @ R      # R^T n as rows
    sd2[:, 4:7] = sd[:, 4:7] @ R
    f2 = po.ff_approx_triangle(sd2, qx, qy, qz, None)
    np.testing.assert_allclose(f1, f2, rtol=1e-12, atol=1e-12 * np.abs(f1).max())


def test_icosphere_approaches_analytic_sphere(po):
    from hipgisaxs_b200 import meshes
    rng = np.random.default_rng(5)
    q = rng.normal(size=(200, 3))
    q *= (rng.uniform(0.05, 0.6, 200) / np.linalg.norm(q, axis=1))[:, None]
    qz = q[:, 2] + 0j
    ana = po.ff_analytic_arrays("sphere", [dict(type="radius", min=10, max=10)], q[:, 0], q[:, 1],
                                qz)
    errs = []
    for sub in (2, 3, 4):
        V, F = meshes.icosphere(10.0, sub)
        sd = po.mesh_to_shape_def(V, F)
        num = po.ff_approx_triangle(sd, q[:, 0], q[:, 1], qz, None)
        # the sphere FF carries exp(i qz R) (origin at the sphere's bottom); the mesh is centred
        errs.append(po.rel_err(np.abs(num), np.abs(ana)))
    assert errs[0] > errs[1] > errs[2]
    assert errs[2] < 2e-2


def test_param_distribution_reference_stepping(po):
    d, w = po.param_distribution("gaussian", 4.25, 5.75, 5.0, 0.25, 7)
    assert len(d) in (6, 7) and d[0] == 4.25
    assert np.all(np.diff(d) > 0)
    d, w = po.param_distribution("none", 5.0, 5.0, 5.0, 0.0, 1)
    assert list(d) == [5.0] and list(w) == [1.0]


def test_dwba_combine_born_limit(po):
    rng = np.random.default_rng(1)
    n = 50
    ff = rng.normal(size=4 * n) + 1j * rng.normal(size=4 * n)
    sf = np.ones(4 * n, complex)
    fc = np.zeros(4 * n, complex)
    fc[:n] = 1.0
    inten = po.dwba_combine(fc, sf, ff, 2.0)
    np.testing.assert_allclose(inten, np.abs(2.0 * ff[:n]) ** 2, rtol=1e-14)


def test_chi2_definition(po):
    m = np.array([1.0, 2.0, 3.0, 0.5])
    c = np.array([1.0, 0.0, 4.0, 9.0])
    mask = np.array([1, 1, 0, 1], np.uint32)
    ref = (2 - 1) ** 2 / 1 + (4 - 0) ** 2 / 1 + (1 - 9) ** 2 / 9
    assert abs(po.chi2(m, c, mask, 2.0) - ref) < 1e-14


def test_normalize_definition(po):
    """HipGISAXS::normalize: (x - min)/(max - min) for all but the first element, which the
    reference leaves as it is; a flat array is left unchanged."""
    x = np.array([5.0, 2.0, 7.0, 4.5])
    d, ok = po.normalize(x)
    assert ok and d[0] == 5.0 and np.allclose(d[1:], (x[1:] - 2.0) / 5.0)
    d, ok = po.normalize(np.full(5, 3.0))
    assert not ok and np.all(d == 3.0)


def test_smearing_preserves_constants_and_is_local(po):
    """Normalised weights: a constant image stays constant; a point spreads no further than
    ceil(6 sigma) pixels."""
    img = np.full((20, 30), 2.5)
    np.testing.assert_allclose(po.smear_gaussian(img, 1.3), img, rtol=1e-14)
    pt = np.zeros((41, 41))
    pt[20, 20] = 1.0
    out = po.smear_gaussian(pt, 1.0)
    nz = np.argwhere(out > 0)
    assert nz.min() >= 20 - 6 and nz.max() <= 20 + 6


def test_structure_sum_rescales_iratios(po):
    I = np.array([[1.0, 2.0], [3.0, 5.0]])
    np.testing.assert_allclose(po.structure_sum(I, [1.0, 3.0]), 0.25 * I[0] + 0.75 * I[1])
    np.testing.assert_allclose(po.structure_sum(I, [0.5, 0.5]), 0.5 * (I[0] + I[1]))
