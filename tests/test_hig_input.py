"""HiG input reader (hgx_hig_read) against the reference's own reader.

The fixtures under tests/golden/hig/ are read by both: <name>.ref.json holds the object model
the reference's HiGInput::construct_input_config builds (tests/golden/hig/gen_hig_golden.py,
oracle/_ref/libhigref.so), and every file under bad/ is rejected by it.  Where the reference
tree is present the reference's own example inputs are compared live as well.  Parsing is
host work: these tests need no GPU.
"""
import ctypes
import glob
import json
import math
import os
import subprocess

import pytest

from conftest import ROOT
from hipgisaxs_b200 import HgxError
from hipgisaxs_b200.hig import read_hig

HIG = os.path.join(ROOT, "tests", "golden", "hig")
FIXTURES = sorted(glob.glob(os.path.join(HIG, "*.hig")))
BAD = sorted(glob.glob(os.path.join(HIG, "bad", "*.hig")))


def model_diff(mine, ref, path=""):
    """Differences between the reader's JSON and the reference's.  The reference leaves some
    fields uninitialised until a file sets them; it reports those under *_raw keys and only
    the ones the file set (present in `mine`) are compared."""
    ref = dict(ref)
    mine = dict(mine)
    out = []
    raw = ref.pop("saveff_savesf_raw", None)
    comp = dict(mine.get("computation", {}))
    if raw is not None:
        for i, k in enumerate(("saveff", "savesf")):
            if k in comp and bool(raw[i]) != comp[k]:
                out.append(f"/computation/{k}: mine={comp[k]} ref={bool(raw[i])}")
            comp.pop(k, None)
        mine["computation"] = comp
    rd = ref.pop("referencedata_raw", None)
    if "referencedata" in mine:
        if rd is None:
            out.append("/referencedata: only in mine")
        else:
            for k, v in mine.pop("referencedata").items():
                if rd.get(k) != v:
                    out.append(f"/referencedata/{k}: mine={v!r} ref={rd.get(k)!r}")
    elif rd is not None:
        out.append("/referencedata: only in the reference")
    algos = ref.pop("algorithms_raw", [])
    mine_algos = mine.pop("algorithms", [])
    if len(algos) != len(mine_algos):
        out.append(f"/algorithms: {len(mine_algos)} in mine, {len(algos)} in the reference")
    else:
        for i, (a, b) in enumerate(zip(mine_algos, algos)):
            for k, v in a.items():
                if b.get(k) != v:
                    out.append(f"/algorithms[{i}]/{k}: mine={v!r} ref={b.get(k)!r}")
    # paracrystal / Percus-Yevick values are compared where the file set them
    for key, st in mine.get("structures", {}).items():
        rs = ref.get("structures", {}).get(key)
        if rs is None:
            continue
        rs = dict(rs)
        st = dict(st)
        for kind in ("paracrystal", "percusyevick"):
            r = rs.pop(kind + "_raw", None)
            m = st.pop(kind, None)
            if m is not None:
                for k, v in m.items():
                    if r is None or r.get(k) != v:
                        out.append(f"/structures/{key}/{kind}/{k}: mine={v!r} ref={None if r is None else r.get(k)!r}")
            elif r is not None:
                out.append(f"/structures/{key}/{kind}: only in the reference")
        mine.setdefault("_st", {})[key] = st
        ref.setdefault("_st", {})[key] = rs
    mine.pop("structures", None)
    ref.pop("structures", None)
    return out + _diff(mine, ref, path)


def _diff(a, b, path):
    out = []
    if isinstance(a, dict) and isinstance(b, dict):
        for k in sorted(set(a) | set(b)):
            if k not in a or k not in b:
                out.append(f"{path}/{k}: only in {'mine' if k in a else 'the reference'}")
            else:
                out += _diff(a[k], b[k], f"{path}/{k}")
    elif isinstance(a, list) and isinstance(b, list) and len(a) == len(b):
        for i, (x, y) in enumerate(zip(a, b)):
            out += _diff(x, y, f"{path}[{i}]")
    elif a != b:
        out.append(f"{path}: mine={a!r} ref={b!r}")
    return out


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p) for p in FIXTURES])
def test_fixture_matches_reference_model(path):
    with open(path[:-4] + ".ref.json") as f:
        ref = json.load(f)
    mine = read_hig(path).data
    d = model_diff(mine, ref)
    assert not d, "\n".join(d)


@pytest.mark.parametrize("path", BAD, ids=[os.path.basename(p) for p in BAD])
def test_rejected_like_the_reference(path):
    with pytest.raises(HgxError) as e:
        read_hig(path)
    assert e.value.status == 1
    assert os.path.basename(path) in str(e.value)  # the message names the file and line


def test_quirks_kept(tmp_path):
    """The reference behaviours the reader reproduces on purpose, one by one."""
    d = read_hig(os.path.join(HIG, "full_grammar.hig"))
    s = d.shapes
    # a shape without refindex keeps the previous shape's (the second "bx" block follows "mesh")
    assert s["bx"]["refindex"] == s["mesh"]["refindex"] == [1e-05, 1e-07]
    # a second shape with the same key merges parameters (Shape::operator=)
    assert sorted(s["bx"]["params"]) == ["edge", "unknownparam", "xsize"]
    assert s["bx"]["params"]["unknownparam"]["type"] == "error"
    assert s["bx"]["params"]["unknownparam"]["stat"] == "error"
    assert s["cyl"]["params"]["height"]["stat"] == "none"  # "single" is stat_none
    assert s["mesh"]["name"] == "custom" and s["mesh"]["name_str"] == "particle.obj"
    assert s["cyl"]["rot"] == [math.pi / 6, -12.5 * math.pi / 180, math.pi / 2]
    # alphai's step also sets the in-plane rotation step
    assert d.scattering_alphai() == (0.12, 0.2, 0.02)
    assert d.scattering_inplanerot() == (0.0, 0.0, 0.02)
    # the second element with the same shape key replaces the first one's locations
    assert d.unitcells["redo"] == {"cyl": [[2, 2, 2], [3, 3, 3]]}
    # orientation extras carry over to the next structure; angles and axes do not
    st = d.structures
    assert st["second"]["rot1"]["mean"] == 5 and st["second"]["rot1"]["sd"] == 2.5
    assert st["second"]["rot2"]["location"] == 1.25 and st["second"]["rot2"]["axis"] == "y"
    assert st["second"]["rot3"]["angles"] == [0, 0]
    # the repetition distribution carries over as well
    assert st["second"]["xrepetition"] == {"stat": "uniform", "min": 2, "max": 9}
    # the grain's layer order stays 0 whatever layer:key says
    assert st["first"]["layer_key"] == "film" and st["first"]["layer_order"] == 0
    # numbers truncated where the reference stores integers
    assert d.layers[2]["order"] == 2 and d.param_resolution() == [64, 33]
    # lattice vectors: table values, fco basis, and no vectors for cubic/111
    assert st["first"]["lattice"]["b"] == [0.5, math.sqrt(3.0) / 2.0, 0]  # hex, any hkl
    assert st["third"]["lattice"]["t"] == [0.5, 0, 0.5]
    assert st["fifth"]["lattice"]["a"] == [1, 0, 0] and st["fifth"]["lattice"]["c"] == [0, 0, 1]
    assert st["second"]["lattice"]["abc_set"] and st["second"]["lattice"]["c"] == [0, 0.5, 1]
    assert st["second"]["scaling_mean"] == [17.5, 17.5, 17.5]
    assert st["second"]["scaling_stddev"] == [0, 0.25, 0] and st["second"]["scaling_nsamples"] == [40, 11, 40]
    # the second algorithm starts from the first one's settings
    a = d.algorithms
    assert a[1]["name"] == "pounders" and a[1]["tolerance"] == 1e-4 and a[1]["order"] == 1
    assert a[1]["params"] == {"pounders_delta": 0.1}
    assert d.compute["saveff"] is True and d.compute["savesf"] is False


def test_beam():
    """k0 = 2 pi / lambda, lambda = 1.23984 / E[keV] (HipGISAXS::init)."""
    d = read_hig(os.path.join(HIG, "paracrystal.hig"))
    k0, ai, _ = d.beam()
    assert k0 == 2 * 3.141592653589793 / (1.23984 / (10000 / 1000))
    assert ai == 0.16 * 3.141592653589793 / 180
    d = read_hig(os.path.join(HIG, "full_grammar.hig"))
    k0, _, _ = d.beam()
    assert k0 == 2 * 3.141592653589793 / (1.23984 / 11.9)


def test_include_found_from_another_directory(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    d = read_hig(os.path.join(HIG, "include_main.hig"))
    assert d.shapes["s1"]["params"]["height"]["min"] == 7


def test_missing_file():
    with pytest.raises(HgxError) as e:
        read_hig(os.path.join(HIG, "no_such_file.hig"))
    assert "cannot open" in str(e.value)


def _reference_tree():
    env = dict(os.environ)
    env.pop("CC", None)
    env.pop("CXX", None)
    ref = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "print-ref"],
                         capture_output=True, text=True, env=env).stdout.strip()
    lib = os.path.join(ROOT, "oracle", "_ref", "libhigref.so")
    if not ref or not os.path.isdir(os.path.join(ref, "examples")) or not os.path.exists(lib):
        pytest.skip("reference tree or oracle/_ref not present")
    return ref, lib


def test_reference_examples_live():
    """The reference's own example inputs, read by both readers here."""
    ref, lib = _reference_tree()
    L = ctypes.CDLL(lib)
    L.ref_hig_json.restype = ctypes.c_long
    L.ref_hig_json.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_long]
    buf = ctypes.create_string_buffer(1 << 22)
    examples = sorted(glob.glob(os.path.join(ref, "examples", "*.hig")))
    assert examples
    for path in examples + FIXTURES:
        cwd = os.getcwd()
        os.chdir(os.path.dirname(path))
        try:
            n = L.ref_hig_json(os.fsencode(path), buf, len(buf))
        finally:
            os.chdir(cwd)
        assert n > 0, path
        d = model_diff(read_hig(path).data, json.loads(buf.value.decode()))
        assert not d, path + "\n" + "\n".join(d)


def test_fit_update_matches_reference():
    """HiGInput::update_params for 51 variables of every form (shape parameters and origin,
    layers, lattice, scaling, translation, repetition, ensemble, orientations, instrument,
    no-op fields and the reference's quirks), against the reference's own update."""
    path = os.path.join(HIG, "fit_update.hig")
    d = read_hig(path)
    keys = d.fit_keys()
    assert keys == sorted(keys) and len(keys) == 51
    d.fit_update([1.5 + 0.25 * i for i in range(len(keys))])
    with open(path[:-4] + ".updated.ref.json") as f:
        ref = json.load(f)
    diff = model_diff(d.data, ref)
    assert not diff, "\n".join(diff)
    s = d.structures["st1"]
    assert d.shapes["cyl"]["originvec"][2] == 1.5 + 0.25 * 7   # "key:z" sets the origin
    assert s["rot2"]["angles"][0] == 1.5 + 0.25 * 32           # rot2's "max" sets its minimum
    assert s["rot3"]["mean"] == 1.5 + 0.25 * 33                # anglemean, then min leaves it


def test_update_param_errors():
    d = read_hig(os.path.join(HIG, "fit_update.hig"))
    for var in ("shape['cyl']:xrot", "shape['nope']:zrot", "structure['st1']:ensemble:spacing:2",
                "structure['st1']:ensemble:orientations:rot1['x']:min", "shape[cyl]:zrot",
                "shape['cyl']:param['width']:min", "detector:sdd"):
        with pytest.raises(HgxError):
            d.update_param(var, 1.0)
    d.update_param("shape['cyl']:zrot", 0.25)  # radians, as the reference takes them
    assert d.shapes["cyl"]["rot"][0] == 0.25


def test_fit_metrics_restatement_is_the_reference():
    """The oracle's restatement of the fitter's eight distance measures against the
    reference's classes (distance_functions.hpp), bit for bit, with masks, zeros and NaNs."""
    import numpy as np
    import pyoracle as po
    if not po.available("ref"):
        pytest.skip("oracle/_ref not built")
    rng = np.random.default_rng(5)
    n = 4000
    ref = rng.gamma(2.0, 3.0, n)
    dat = rng.gamma(2.0, 3.0, n)
    ref[:10] = 0
    dat[10:20] = 0
    ref[20:25] = -1.0
    mask = (rng.random(n) > 0.1).astype(np.uint32)
    for name in po.FIT_METRICS:
        for mk in (None, mask):
            a = po.fit_distance(name, ref, dat, mk, "port")
            b = po.fit_distance(name, ref, dat, mk, "ref")
            assert np.array_equal(a, b, equal_nan=True), name


def test_fit_update_live_against_reference():
    _, lib = _reference_tree()
    import importlib.util
    spec = importlib.util.spec_from_file_location("gen_hig", os.path.join(HIG, "gen_hig_golden.py"))
    gen = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gen)
    path = os.path.join(HIG, "fit_update.hig")
    d = read_hig(path)
    keys = d.fit_keys()
    vals = [0.75 - 0.5 * i for i in range(len(keys))]
    d.fit_update(vals)
    diff = model_diff(d.data, gen.ref_updated(path, keys, vals))
    assert not diff, "\n".join(diff)


def test_scan_points_follow_the_reference_loops(tmp_path):
    """run_all_gisaxs's scan counts ((max - min) / step + 1 truncated; 1 for a zero step;
    alphai's max raised to its min) and its angles accumulated from the minimum, alpha_i
    outermost and tilt innermost."""
    d = read_hig(os.path.join(HIG, "sim_scan.hig"))
    assert d.scan_size() == (3, 3, 2)
    want, a = [], 0.12
    for _ in range(3):
        p = 0.0
        for _ in range(3):
            t = 0.0
            for _ in range(2):
                want.append((a, p, t))
                t += 1.0
            p += 15.0
        a += 0.04
    assert d.scan_points() == want
    text = open(os.path.join(HIG, "sim_scan.hig")).read()
    for old, new, size in [
        ("alphai = { min = 0.12, max = 0.2, step = 0.04 }", "alphai = { min = 0.12, max = 0.05, step = 0.04 }", (1, 3, 2)),
        ("inplanerot = { min = 0, max = 30, step = 15 }", "inplanerot = { min = 30, max = 0, step = 15 }", (3, 0, 2)),
        ("tilt = { min = 0, max = 1, step = 1 }", "tilt = { min = 0, max = 1, step = 0 }", (3, 3, 1)),
    ]:
        p = tmp_path / "s.hig"
        p.write_text(text.replace(old, new))
        e = read_hig(str(p))
        assert e.scan_size() == size
        assert len(e.scan_points()) == size[0] * size[1] * size[2]
    from hipgisaxs_b200._capi import check, lib
    for p in (-1, 18):
        with pytest.raises(HgxError):
            check(lib().hgx_hig_scan_point(d.handle, p, None, None, None))
