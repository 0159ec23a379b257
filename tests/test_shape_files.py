"""Shape-definition files: the OBJ reader (ObjectShapeReader::load_object semantics, no Boost)
and read_shapes_file (.obj through the device triangle conversion, raw .dat), against the
oracle's restatement of get_triangle_params / convert_to_shape."""
import ctypes as C

import numpy as np
import pytest

import hipgisaxs_b200 as hg
from hipgisaxs_b200 import _capi, meshes


def _mixed_obj(tmp_path):
    """An icosphere written with every face-item form, CRLF endings, comments, ignored
    statements, a quad, a pentagon and a degenerate triangle."""
    V, F = meshes.icosphere(7.0, 1)
    V = np.vstack([V, [[1.0, 1.0, 1.0]]])           # extra vertex for a degenerate face
    forms = ["{a}", "{a}/{t}", "{a}/{t}/{n}", "{a}//{n}"]
    lines = ["# test mesh", "mtllib x.mtl", "o ball", "g part", "s 1", "usemtl m", ""]
    lines += [f"v {x:.17g}\t{y:.17g}  {z:.17g}" for x, y, z in V]
    lines += ["vt 0.5 0.5", "vn 0 0 1", "l 1 2"]
    for i, (a, b, c) in enumerate(F):
        fm = forms[i % 4]
        items = [fm.format(a=k + 1, t=1, n=1) for k in (a, b, c)]
        lines.append("f " + " ".join(items))
    lines.append("f 1 2 3 4")                        # quad: left out
    lines.append("f 1 2 3 4 5")                      # pentagon: skipped
    d = len(V)
    lines.append(f"f {d} {d} {d}")                   # degenerate: kept by the reader
    p = tmp_path / "mixed.obj"
    p.write_bytes(("\r\n".join(lines) + "\r\n").encode())
    Fall = np.vstack([F, [[d - 1, d - 1, d - 1]]])
    return p, V, Fall


def test_obj_reader_forms_and_counts(tmp_path):
    p, V, F = _mixed_obj(tmp_path)
    v, f, info = meshes.load_obj(p)
    np.testing.assert_array_equal(v, V)
    np.testing.assert_array_equal(f, F)
    assert info == {"nquads": 1, "nskipped": 1}


def test_obj_reader_round_trip(tmp_path):
    V, F = meshes.icosphere(10.0, 2)
    p = tmp_path / "ico.OBJ"
    meshes.write_obj(p, V, F)
    v, f, info = meshes.load_obj(p)
    np.testing.assert_array_equal(v, V)
    np.testing.assert_array_equal(f, F)
    assert info == {"nquads": 0, "nskipped": 0}


@pytest.mark.parametrize("body", ["v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 4\n",   # out of range
                                  "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 -1\n",  # relative index
                                  "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 x\n",   # not an integer
                                  "v 0 0 0\nv 1 0\n",                       # short vertex
                                  "v 0 0 0\nf 1/2/3/4 1 1\n"])              # too many slashes
def test_obj_reader_rejects_malformed(tmp_path, body):
    p = tmp_path / "bad.obj"
    p.write_text(body)
    with pytest.raises(hg.HgxError):
        meshes.load_obj(p)


def test_obj_reader_missing_file(tmp_path):
    with pytest.raises(hg.HgxError):
        meshes.load_obj(tmp_path / "none.obj")


def test_dat_shapes_file_without_gpu(tmp_path):
    rng = np.random.default_rng(3)
    rows = rng.normal(size=(17, 7))
    p = tmp_path / "tri.dat"
    # 17 records and a trailing incomplete one, which ends the file as in the reference
    p.write_text("\n".join(" ".join(f"{x:.17g}" for x in r) for r in rows) + "\n1 2 3\n")
    out = meshes.read_shapes_file(None, p)   # the raw reader does no device work
    assert out.shape == (17, 8)
    np.testing.assert_array_equal(out[:, :7], rows)
    assert np.all(out[:, 7] == 0)


def test_unknown_and_hdf5_formats_rejected(tmp_path):
    n = C.c_int()
    for name in ("shape.hd5", "shape.HDF5", "shape.stl", "noext"):
        (tmp_path / name).write_text("")
        s = _capi.lib().hgx_read_shapes_file(None, str(tmp_path / name).encode(), None, 0,
                                             C.byref(n))
        assert s != 0


def test_obj_file_needs_a_context(tmp_path):
    V, F = meshes.icosphere(5.0, 1)
    p = tmp_path / "a.obj"
    meshes.write_obj(p, V, F)
    with pytest.raises(hg.HgxError):
        meshes.read_shapes_file(None, p)


@pytest.mark.gpu
def test_obj_shapes_file_matches_oracle(ctx, po, tmp_path):
    p, V, F = _mixed_obj(tmp_path)
    sd = meshes.read_shapes_file(ctx, p)
    ref = po.mesh_to_shape_def(V, F)          # convert_to_shape: degenerate faces dropped
    assert sd.shape == ref.shape == (len(F) - 1, 8)
    np.testing.assert_allclose(sd, ref, rtol=1e-14, atol=1e-14)
    # and the form factor of the file equals that of the in-memory mesh
    G = po.Grid(16, 12, -1.0, 0.0, 1.0, 2.0, 0.16, 10.0)
    g = hg.QGrid.from_arrays(ctx, G.qx, G.qy, G.qz_ext)
    a = hg.ff_triangles(ctx, g, sd, None, "f64")
    assert po.rel_err(a, po.ff_approx_triangle(ref, G.qx, G.qy, G.qz_ext)) < 1e-12
