"""Host-side logic of the C ABI that runs without a GPU: the reference's parameter sampling
and lattice table, checked against the oracle."""
import numpy as np
import pytest

from hipgisaxs_b200 import model


@pytest.mark.parametrize("case", [
    ("gaussian", 4.25, 5.75, 5.0, 0.25, 11), ("uniform", 3.0, 5.0, float("nan"), 0.0, 3),
    ("none", 5.0, 5.0, 5.0, 0.0, 1), ("gaussian", 8.5, 11.5, float("nan"), 0.5, 7),
    ("uniform", 1.0, 2.0, 0.0, 0.0, 10)])
def test_param_distribution_matches_oracle(po, case):
    v, w = model.param_distribution(*case)
    ov, ow = po.param_distribution(*case)
    np.testing.assert_array_equal(v, ov)
    np.testing.assert_allclose(w, ow, rtol=1e-15)


@pytest.mark.parametrize("kind,hkl", [("hex", "100"), ("cubic", "100"), ("cubic", "110"),
                                      ("bcc", "100"), ("bcc", "110"), ("fcc", "100"),
                                      ("fcc", "111"), ("fco", "100"), ("hcp", "100")])
def test_lattice_vectors_match_oracle(po, kind, hkl):
    abc, t = model.lattice_vectors(kind, hkl)
    oa, ob, oc, ot = po.lattice_vectors(kind, hkl)
    np.testing.assert_array_equal(abc, np.array([oa, ob, oc]))
    np.testing.assert_array_equal(t, ot)


def test_lattice_vectors_reject_unknown():
    from hipgisaxs_b200 import HgxError
    with pytest.raises(HgxError):
        model.lattice_vectors("cubic", "111")


def test_save_gisaxs_matches_the_stream_format(tmp_path):
    """The ".out" text of HipGISAXS::save_gisaxs: default C++ stream formatting (6 significant
    digits, %g-like), a tab after every value, one row per line."""
    from hipgisaxs_b200 import model
    img = np.array([[1.0, 2.5e-7, 123456789.0], [0.0, -3.25, 1e5], [7e-5, 42.0, 1.0 / 3.0]])
    p = tmp_path / "img.out"
    model.save_gisaxs(p, img)
    expect = "".join("".join(f"{v:g}\t" for v in row) + "\n" for row in img)
    assert p.read_text() == expect
