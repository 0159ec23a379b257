"""HiG-driven device set-up (hgx_hig_qgrid) against the oracle's QGrid::create."""
import os

import numpy as np
import pytest

from conftest import ROOT
import hipgisaxs_b200 as hg
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
       "sim_orientations.hig", "sim_shapes.hig", "sim_mesh_paracrystal.hig", "sim_saxs.hig",
       "sim_saxs_py.hig"]


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
def test_compute_gisaxs_mesh_kept_until_file_changes(ctx, po, tmp_path):
    """The custom shape's triangles stay on the device between calls and are read again when
    the shape file changes: each image equals the oracle's for the file as it is then."""
    import shutil
    import time
    shutil.copy(os.path.join(HIG, "sim_two_structures.hig"), tmp_path / "m.hig")
    obj = tmp_path / "octahedron.obj"
    shutil.copy(os.path.join(HIG, "octahedron.obj"), obj)
    d = read_hig(str(tmp_path / "m.hig"))

    def both():
        _srand(5)
        img = d.compute_gisaxs(ctx)
        _srand(5)
        ref = po.compute_gisaxs(d.data, str(tmp_path))
        assert np.abs(img - ref).max() / np.abs(ref).max() < 1e-11
        return img

    a = both()
    np.testing.assert_array_equal(both(), a)  # the kept triangles
    lines = []
    for ln in obj.read_text().splitlines():
        if ln.startswith("v "):
            x, y, z = (float(t) * 1.3 for t in ln.split()[1:4])
            ln = f"v {x!r} {y!r} {z!r}"
        lines.append(ln)
    obj.write_text("\n".join(lines) + "\n")
    st = os.stat(obj)
    os.utime(obj, ns=(st.st_atime_ns, st.st_mtime_ns + 5_000_000_000))
    b = both()
    assert np.abs(b - a).max() > 1e-3 * np.abs(a).max()


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
@pytest.mark.parametrize("precision", ["f64", "f32c"])
def test_device_images_back_to_back(ctx, precision):
    """With a device image a simulation returns once its work is queued, so the host stages the
    next one's tables (alternating pinned arenas) while earlier ones still run.  Five
    simulations in a row with different fit parameters into five device images, synchronised
    once at the end, equal the same simulations with host images (each synchronous)."""
    torch = pytest.importorskip("torch")
    d = read_hig(os.path.join(HIG, "fit_objective.hig"))
    nrow, ncol = d.image_size()
    xs = [[4.0, 22.0, 5.0], [5.5, 25.0, 12.0], [3.5, 19.0, 0.0], [6.0, 28.0, 20.0], [4.2, 21.0, 0.3]]
    outs = [torch.full((nrow * ncol,), -1.0, dtype=torch.float64, device="cuda:0") for _ in xs]
    for x, out in zip(xs, outs):
        d.fit_update(x)
        d.compute_gisaxs(ctx, precision=precision, out=out)
    ctx.synchronize()
    for x, out in zip(xs, outs):
        d.fit_update(x)
        host = d.compute_gisaxs(ctx, precision=precision)
        assert np.array_equal(out.cpu().numpy().reshape(nrow, ncol), host)
    d.close()


@pytest.mark.gpu
def test_device_images_across_a_stream_change(ctx):
    """An asynchronous simulation queued on one stream, then the context moved to another
    stream and a second simulation queued there: the change of stream waits for the first, so
    both images equal their synchronous host-image versions."""
    torch = pytest.importorskip("torch")
    d = read_hig(os.path.join(HIG, "fit_objective.hig"))
    nrow, ncol = d.image_size()
    c2 = hg.Context(0)
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    a = torch.full((nrow * ncol,), -1.0, dtype=torch.float64, device="cuda:0")
    b = torch.full((nrow * ncol,), -1.0, dtype=torch.float64, device="cuda:0")
    torch.cuda.synchronize()
    c2.set_stream(s1)
    d.fit_update([5.5, 25.0, 12.0])
    d.compute_gisaxs(c2, out=a)
    c2.set_stream(s2)
    d.fit_update([3.5, 19.0, 0.0])
    d.compute_gisaxs(c2, out=b)
    c2.synchronize()
    got_a, got_b = a.cpu().numpy().reshape(nrow, ncol), b.cpu().numpy().reshape(nrow, ncol)
    c2.set_stream(None)
    d.fit_update([5.5, 25.0, 12.0])
    want_a = d.compute_gisaxs(c2)
    d.fit_update([3.5, 19.0, 0.0])
    want_b = d.compute_gisaxs(c2)
    assert np.array_equal(got_a, want_a) and np.array_equal(got_b, want_b)
    c2.close()
    d.close()


@pytest.mark.gpu
@pytest.mark.parametrize("edit,words", [
    (("scattering = {", 'scattering = { expt = "waxs",'), "experiment"),
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


@pytest.mark.gpu
def test_fit_distance_matches_oracle(ctx, po):
    """hgx_fit_distance against the oracle's restatement (itself the reference's classes, bit
    for bit): 1e-12 relative for the sums (the device sums run in another order)."""
    from hipgisaxs_b200.hig import METRICS, fit_distance
    rng = np.random.default_rng(9)
    n = 70_001
    ref = rng.gamma(2.0, 3.0, n)
    dat = rng.gamma(2.0, 3.0, n)
    ref[:10] = 0
    dat[10:20] = 0
    mask = (rng.random(n) > 0.1).astype(np.uint32)
    for name in METRICS:
        for mk in (None, mask):
            got = fit_distance(ctx, name, ref, dat, mk)
            want = po.fit_distance(name, ref, dat, mk)
            assert got.shape == want.shape, name
            # per-pixel residual terms |n_d - n_r|^2 cancel where model and reference agree:
            # there the norms' summation order shows, so they are held to 1e-12 of the largest
            np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12 * np.abs(want).max(),
                                       err_msg=name)


@pytest.mark.gpu
@pytest.mark.parametrize("metric", ["sqrt_unit_l2", "sqrt_c_l2", "cbrt_c_l2", "sqrt_unit_l2_residual"])
def test_objective_matches_oracle(ctx, po, metric):
    """HipGISAXSObjectiveFunction::operator()(x) for a HiG fitting block: the parameters set in
    key order, the simulation, the distance to a reference image and the regularisation,
    against the oracle's composition of the same steps."""
    d = read_hig(os.path.join(HIG, "fit_objective.hig"))
    assert d.fit_keys() == ["radius", "spacing", "twist"]
    d.fit_update([5.0, 25.0, 12.0])
    ref_img = po.compute_gisaxs(d.data, HIG)
    mask = np.ones(ref_img.size, dtype=np.uint32)
    mask[::7] = 0
    x = [4.2, 21.0, 3.0]
    alpha = 0.5
    got = d.objective(ctx, x, ref_img, mask, metric, alpha)
    # the oracle on the same updated description
    img = po.compute_gisaxs(d.data, HIG)
    want = po.fit_distance(metric, ref_img, img, mask)
    means = [(7 + 3) / 2.0, (30 + 18) / 2.0, (30 + 0) / 2.0]
    reg = (alpha / 2) * sum((xi - m) ** 2 for xi, m in zip(x, means))
    want = np.where(np.isfinite(want), want + reg / want.size, 1e8)
    assert got.shape == want.shape
    np.testing.assert_allclose(got, want, rtol=1e-10, atol=0)


@pytest.mark.gpu
def test_scan_points_match_oracle(ctx, po):
    """run_all_gisaxs's scan on the device, point by point, against the oracle's composition
    at each point's alpha_i and phi (grid of the first alpha_i, qz_extended and Fresnel
    coefficients at the point's); the rand()-drawn orientations continue across points on
    both sides.  The per-alpha_i sums over phi and tilt are the reference's "averaged" output."""
    d = read_hig(os.path.join(HIG, "sim_scan.hig"))
    pts = d.scan_points()
    _srand(21)
    images, sums = d.run_all_gisaxs(ctx)
    _srand(21)
    refs = [po.compute_gisaxs(d.data, HIG, alpha_i=a, phi=p) for a, p, _ in pts]
    assert len(images) == len(refs) == 18
    for (a, p, t, img), ref in zip(images, refs):
        assert np.abs(img - ref).max() / np.abs(ref).max() < 1e-11, (a, p, t)
    assert sorted(sums) == sorted({a for a, _, _ in pts})
    for a in sums:
        want = sum(ref for (pa, _, _), ref in zip(pts, refs) if pa == a)
        assert np.abs(sums[a] - want).max() / np.abs(want).max() < 1e-11
    # a different incidence angle changes the image; the first point equals compute_gisaxs of
    # the description without scans
    assert np.abs(images[0][3] - images[6][3]).max() > 1e-6 * np.abs(images[0][3]).max()
    text = open(os.path.join(HIG, "sim_scan.hig")).read()
    one = text.replace("alphai = { min = 0.12, max = 0.2, step = 0.04 }, inplanerot = { min = 0, max = 30, "
                       "step = 15 }, tilt = { min = 0, max = 1, step = 1 }", "alphai = { min = 0.12 }")
    assert one != text
    import tempfile
    with tempfile.TemporaryDirectory() as tdir:
        p1 = os.path.join(tdir, "one.hig")
        with open(p1, "w") as f:
            f.write(one)
        e = read_hig(p1)
        _srand(21)
        first = e.compute_gisaxs(ctx)
    np.testing.assert_array_equal(first, images[0][3])


@pytest.mark.gpu
def test_sliced_layers_give_the_reference_empty_image(ctx, tmp_path):
    """nslices > 1: run_gisaxs's slicing branch only prints that it is not implemented and adds
    nothing (src/sim/hipgisaxs_main.cpp:1106-1115), so the image is zero; the orientations are
    still drawn, so rand() is left where the reference leaves it."""
    import ctypes
    libc = ctypes.CDLL(None)
    text = open(os.path.join(HIG, "sim_cylinders_hcp.hig")).read()
    p = tmp_path / "sliced.hig"
    p.write_text(text.replace("resolution = [ 48 32 ]", "resolution = [ 48 32 ], nslices = 3", 1))
    d = read_hig(str(p))
    libc.srand(4)
    img = d.compute_gisaxs(ctx)
    after = libc.rand()
    assert img.shape == d.image_size() and not img.any()
    # the same description unsliced draws the same orientations
    libc.srand(4)
    full = read_hig(os.path.join(HIG, "sim_cylinders_hcp.hig")).compute_gisaxs(ctx)
    assert libc.rand() == after and full.max() > 0


# Descriptions whose unit cells hold one cylinder, sphere or box shape on a DWBA grid with
# real qz: the fused grain kernel's FP32C bodies (FP64 phases, FP32 transcendentals and sums).
F32C_SIM = ["sim_cylinders_hcp.hig", "paracrystal.hig", "percus_yevick.hig", "sim_scaling.hig",
            "sim_repetition.hig", "sim_orientations.hig"]


@pytest.mark.gpu
@pytest.mark.parametrize("name", F32C_SIM)
def test_compute_gisaxs_f32c_analytic(ctx, po, name):
    """The FP32C grain kernel against the oracle's FP64 composition: norm-wise relative error
    of the image below 1e-5 and every pixel within 1e-5 of the image's largest value; the
    image differs from the FP64 kernel's (the FP32C bodies ran)."""
    d = read_hig(os.path.join(HIG, name))
    _srand(5)
    img = d.compute_gisaxs(ctx, precision="f32c")
    _srand(5)
    img64 = d.compute_gisaxs(ctx, precision="f64")
    _srand(5)
    ref = po.compute_gisaxs(d.data, HIG)
    assert np.all(np.isfinite(img))
    assert po.rel_err(img, ref) < 1e-5
    assert np.abs(img - ref).max() / np.abs(ref).max() < 1e-5
    assert not np.array_equal(img, img64)


# Cylinders (R 5 nm, H 10 nm, 11 samples each over +-3 sigma of a 5 % spread) on a hex lattice
# a = 20 nm with 20 x 20 repetitions over a Si-like substrate, 10 keV, alpha_i 0.20 deg, a
# 1024 x 1024 DWBA detector over qy in [-2, 2], qz in [0, 3] nm^-1: the full DWBA simulation
# that the benchmark times in FP32C and FP64.
CYL_HEX_1024 = """hipGisaxsInput = {
	shape = { key = "cyl", name = "cylinder", refindex = { delta = 4.88E-06, beta = 7.37E-08 },
		param = { type = "radius", stat = "gaussian", min = 4.25, max = 5.75, p1 = 5, p2 = 0.25, nvalues = 11 },
		param = { type = "height", stat = "gaussian", min = 8.5, max = 11.5, p1 = 10, p2 = 0.5, nvalues = 11 } },
	unitcell = { key = "u1", element = { shape:key = "cyl", locations = [[0 0 0]] } },
	layer = { key = "substr", order = -1, refindex = { delta = 4.88E-06, beta = 7.37E-08 } },
	structure = { key = "st1",
		grain = { unitcell:key = "u1", lattice = { type = "hex" }, repetition = [20 20 1], scaling = 20 },
		ensemble = { maxgrains = [1 1 1] } },
	instrumentation = { scattering = { alphai = { min = 0.2 }, photon = { value = 10000, unit = "ev" } },
		detector = { pixelsize = 0.172, sdd = 4000, directbeam = [ 0 0 ] } },
	computation = { runname = "cylhex", outputregion = { type = "qspace", minpoint = [ -2 0 ], maxpoint = [ 2 3 ] },
		resolution = [ 1024 1024 ] }
}
"""


@pytest.mark.gpu
def test_cylinders_on_hex_lattice_full_size(ctx, tmp_path):
    """The full-size DWBA simulation of cylinders on a hex lattice (1024 x 1024): FP32C against
    the FP64 kernel, norm-wise 1e-5 (measured 2.8e-7) and every pixel within 1e-5 of the
    image's largest value (measured 5.9e-7); the FP64 image is finite and not zero."""
    path = tmp_path / "cylhex.hig"
    path.write_text(CYL_HEX_1024)
    d = read_hig(str(path))
    img32 = d.compute_gisaxs(ctx, precision="f32c")
    img64 = d.compute_gisaxs(ctx, precision="f64")
    assert img64.shape == (1024, 1024) and np.all(np.isfinite(img64)) and img64.max() > 0
    assert np.linalg.norm(img32 - img64) / np.linalg.norm(img64) < 1e-5
    assert np.abs(img32 - img64).max() / np.abs(img64).max() < 1e-5
    d.close()


def _oracle_objective(po, d, x, ref_img, mask, metric, alpha):
    d.fit_update(x)
    img = po.compute_gisaxs(d.data, HIG)
    v = po.fit_distance(metric, ref_img, img, mask)[0]
    means = [(fp["range"][1] + fp["range"][0]) / 2.0 for _, fp in sorted(d.fit_params.items())]
    return v + (alpha / 2) * sum((xi - m) ** 2 for xi, m in zip(x, means))


def _richardson(f, x, j, h):
    def central(hh):
        xp, xm = np.array(x, float), np.array(x, float)
        xp[j] += hh
        xm[j] -= hh
        return (f(xp) - f(xm)) / (2 * hh)
    return (4 * central(h / 2) - central(h)) / 3


GRAD_CASES = [("fit_objective.hig", [5.0, 25.0, 12.0], [4.2, 21.0, 0.3]),
              ("fit_grad_shapes.hig", [4.3, 0.5, 6.5, 1.05, 1.5, 1.0, 75.0],
               [4.0, 0.4, 6.0, 1.0, 1.0, 3.0, 70.0])]


@pytest.mark.gpu
@pytest.mark.parametrize("case", range(len(GRAD_CASES)))
@pytest.mark.parametrize("metric", ["sqrt_unit_l2", "sqrt_c_l2", "cbrt_unit_l2", "sqrt_unit_l1"])
def test_objective_gradient_matches_oracle_differences(ctx, po, case, metric):
    """d(objective)/dx by the simulation's tangent (hgx_hig_objective_grad) against Richardson
    central differences of the oracle's objective (FP64), every parameter kind: a cylinder's
    radius, a sphere distribution's mean and width, a box's size, a lattice vector, a grain
    translation, an orientation mean (gaussian weights), a grain scaling and spacing, an
    orientation angle.  Tolerance: 1e-5 of the gradient's norm, component by component."""
    name, xtrue, x = GRAD_CASES[case]
    d = read_hig(os.path.join(HIG, name))
    d.fit_update(xtrue)
    ref_img = po.compute_gisaxs(d.data, HIG)
    mask = np.ones(ref_img.size, dtype=np.uint32)
    mask[::7] = 0
    alpha = 0.3
    f, g = d.objective_grad(ctx, x, ref_img, mask, metric, alpha)
    f0 = d.objective(ctx, x, ref_img, mask, metric, alpha)[0]
    assert abs(f - f0) <= 1e-14 * abs(f0)

    def fo(xx):
        return _oracle_objective(po, d, xx, ref_img, mask, metric, alpha)

    assert abs(fo(x) - f) < 1e-10 * abs(f)
    # a small step: the reference's principal-branch lattice factor has kinks (its slope
    # changes sign where a lattice angle crosses an odd multiple of pi, for even repetitions)
    # and a wide difference straddles them at some pixels
    fd = np.array([_richardson(fo, x, j, 1e-5 * max(1.0, abs(x[j]))) for j in range(len(x))])
    scale = np.linalg.norm(fd)
    assert np.all(np.abs(g - fd) <= 1e-5 * scale), (g, fd)


@pytest.mark.gpu
@pytest.mark.parametrize("case", range(len(GRAD_CASES)))
def test_population_matches_objective_calls(ctx, po, case):
    """hgx_hig_population: every candidate's distance equals hgx_hig_objective's for its
    parameter vector (the same simulation arithmetic and distance sums, one call per particle
    as the reference's PSO loop makes them), on the first evaluation (graph recorded) and on a
    second generation (replayed); the FP32C population within 1e-5 of it."""
    name, xtrue, x0 = GRAD_CASES[case]
    d = read_hig(os.path.join(HIG, name))
    d.fit_update(xtrue)
    ref_img = po.compute_gisaxs(d.data, HIG)
    mask = np.ones(ref_img.size, dtype=np.uint32)
    mask[::5] = 0
    rng = np.random.default_rng(7 + case)
    npop = 6
    pop = d.population(ctx, npop, ref_img, mask, "sqrt_c_l2", 0.2)
    pop32 = d.population(ctx, npop, ref_img, mask, "sqrt_c_l2", 0.2, "f32c")
    for gen in range(2):
        X = np.array(x0) * (1 + rng.uniform(-0.03, 0.03, (npop, len(x0))))
        got, got32 = pop.eval(X), pop32.eval(X)
        for i in range(npop):
            want = d.objective(ctx, X[i], ref_img, mask, "sqrt_c_l2", 0.2)[0]
            assert abs(got[i] - want) <= 1e-12 * abs(want), (gen, i, got[i], want)
            assert abs(got32[i] - want) <= 1e-5 * abs(want), (gen, i, got32[i], want)
    pop.close()
    pop32.close()


@pytest.mark.gpu
def test_population_refusals(ctx):
    d = read_hig(os.path.join(HIG, "fit_objective.hig"))
    ref_img = np.ones(d.image_size())
    with pytest.raises(hg.HgxError):  # the residual vectors are not one value per candidate
        d.population(ctx, 4, ref_img, None, "sqrt_unit_l2_residual")
    d2 = read_hig(os.path.join(HIG, "fit_update.hig"))  # random orientations
    with pytest.raises(hg.HgxError):
        d2.population(ctx, 4, np.ones(d2.image_size()))
    pop = d.population(ctx, 2, ref_img)
    with pytest.raises(hg.HgxError):  # one row per candidate, one value per fit parameter
        lib_x = np.ones((2, len(d.fit_keys()) + 1))
        hg._capi.check(hg.lib().hgx_hig_population_eval(pop._h, lib_x.ctypes.data, lib_x.shape[1],
                                                        np.zeros(2).ctypes.data))
    pop.close()


@pytest.mark.gpu
def test_objective_gradient_refuses_what_it_cannot_differentiate(ctx, po):
    d = read_hig(os.path.join(HIG, "fit_objective.hig"))
    ref_img = np.ones(d.image_size())
    x = [4.2, 21.0, 0.3]
    with pytest.raises(hg.HgxError):  # residual-vector measures have no scalar gradient
        d.objective_grad(ctx, x, ref_img, None, "sqrt_unit_l2_residual")
    d2 = read_hig(os.path.join(HIG, "fit_update.hig"))  # random orientations, iratios, layers
    with pytest.raises(hg.HgxError):
        d2.objective_grad(ctx, [float(v) for v in range(len(d2.fit_keys()))],
                          np.ones(d2.image_size()), None, "sqrt_unit_l2")


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["paracrystal.hig", "percus_yevick.hig"])
def test_population_with_liquid_structure_factors(ctx, po, tmp_path, name):
    """A population over a sphere radius where the structure factor is grain-independent
    (paracrystal, Percus-Yevick: made once at creation and shared by every candidate): each
    distance equals hgx_hig_objective's (1e-12), FP32C within 1e-5."""
    text = open(os.path.join(HIG, name)).read().rstrip().rstrip("}").rstrip()
    text += (',\n\tfitting = {\n\t\tfitparam = { key = "r", variable = "shape[\'sph\']:param[\'radius\']:min", '
             'range = { min = 3, max = 7 }, init = 5 },\n\t\talgorithm = { algoname = "pso", '
             'distancemetric = "sqrt_unit_l2" }\n\t}\n}\n')
    path = tmp_path / name
    path.write_text(text)
    d = read_hig(str(path))
    d.fit_update([5.3])
    ref_img = po.compute_gisaxs(d.data, HIG).ravel()
    X = np.array([[4.1], [4.9], [5.3], [6.2], [6.8]])
    pop = d.population(ctx, len(X), ref_img, None, "sqrt_unit_l2", 0.1)
    pop32 = d.population(ctx, len(X), ref_img, None, "sqrt_unit_l2", 0.1, "f32c")
    got, got32 = pop.eval(X), pop32.eval(X)
    for i, x in enumerate(X):
        want = d.objective(ctx, x, ref_img, None, "sqrt_unit_l2", 0.1)[0]
        assert abs(got[i] - want) <= 1e-12 * abs(want), (i, got[i], want)
        assert abs(got32[i] - want) <= 1e-5 * abs(want), (i, got32[i], want)
    pop.close()
    pop32.close()
