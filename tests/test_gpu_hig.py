"""HiG-driven device set-up (hgx_hig_qgrid) against the oracle's QGrid::create."""
import os

import numpy as np
import pytest

from conftest import ROOT
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
