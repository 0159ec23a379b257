"""Post-processing on the GPU: Gaussian smearing against the golden images made by the
reference's compiled Convolutions::convolution_gaussian_2d and against the oracle, and
normalize against the oracle.  FP64 kernels without fused multiply-adds: expected equal to
the reference within 1e-14 (relative, norm-wise)."""
import numpy as np
import pytest

import hipgisaxs_b200 as hg
from hipgisaxs_b200 import model

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["s07", "s20", "s35"])
def test_smearing_golden(ctx, po, golden, name):
    d = golden(f"smear_{name}")
    got = model.gaussian_smearing(ctx, d["image"], float(d["sigma"]))
    assert po.rel_err(got, d["smeared"]) < 1e-14


def test_smearing_large_image_device_in_place(ctx, po):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(4)
    img = rng.random((300, 517))
    ref = po.smear_gaussian(img, 4.2)
    t = torch.tensor(img, device="cuda:0")
    model.gaussian_smearing(ctx, t, 4.2)
    ctx.synchronize()
    assert po.rel_err(t.cpu().numpy(), ref) < 1e-14


def test_smearing_rejects_bad_sigma(ctx):
    img = np.ones((4, 4))
    for s in (0.0, -1.0, 1e4):
        with pytest.raises(hg.HgxError):
            model.gaussian_smearing(ctx, img, s)


def test_normalize(ctx, po):
    rng = np.random.default_rng(6)
    x = rng.normal(size=1_000_003) * 7.0 + 3.0
    got, ok = model.normalize(ctx, x)
    ref, ok_ref = po.normalize(x)
    assert ok and ok_ref
    np.testing.assert_array_equal(got, ref)
    flat, ok = model.normalize(ctx, np.full(17, 4.0))
    assert not ok and np.all(flat == 4.0)
