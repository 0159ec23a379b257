import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: full-size workloads")


def _ensure_built():
    """Builds the oracle (and the reference oracle where the reference tree exists) once."""
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True,
                       capture_output=True)


_ensure_built()


def assert_exact_ff_close(po, got, tris, qx, qy, qz, rot=None, extra=0.0):
    """Parity check of the exact (polyhedral) triangle form factor, point by point.  The
    reference's formula adds edge and vertex terms of size O(1/(|q|^2 proj_t proj_e)) that
    cancel to O(area) — at small |q| the cancellation is severe, so the reference's own result
    moves by up to O(1) under a relative 1e-15 change of its inputs (its conditioning, not an
    error of either implementation).  Each q-point may therefore differ from the oracle by 10x
    the oracle's own spread under four seeded 1e-15 relative perturbations (two of the vertex
    coordinates, two of the q-vectors), plus 1e-12 (plus `extra`, e.g. an output rounding)
    times the rms of the result.  Returns the fraction of q-points whose spread exceeds 1e-12
    of the rms."""
    tris = np.asarray(tris, dtype=np.float64)
    qx, qy = np.asarray(qx, dtype=np.float64), np.asarray(qy, dtype=np.float64)
    qz = np.asarray(qz, dtype=np.complex128)
    ref = po.ff_exact_triangle(tris, qx, qy, qz, rot)
    spread = np.zeros(len(ref))
    for seed in range(4):
        r = np.random.default_rng(seed)
        if seed < 2:
            args = (tris * (1.0 + 1e-15 * r.standard_normal(tris.shape)), qx, qy, qz)
        else:
            args = (tris, qx * (1.0 + 1e-15 * r.standard_normal(qx.shape)),
                    qy * (1.0 + 1e-15 * r.standard_normal(qy.shape)),
                    qz * (1.0 + 1e-15 * r.standard_normal(qz.shape)))
        spread = np.maximum(spread, np.abs(po.ff_exact_triangle(*args, rot) - ref))
    rms = np.sqrt(np.mean(np.abs(ref) ** 2))
    allowed = 10.0 * spread + (1e-12 + extra) * rms
    err = np.abs(np.asarray(got, dtype=np.complex128) - ref)
    bad = np.flatnonzero(err > allowed)
    assert bad.size == 0, (f"{bad.size} of {len(ref)} q-points beyond the bound; worst "
                           f"{np.max(err[bad] / allowed[bad]):.3g}x at q-point {bad[np.argmax(err[bad] / allowed[bad])]}")
    return float(np.mean(spread > 1e-12 * rms))


@pytest.fixture(scope="session")
def po():
    import pyoracle
    pyoracle.set_threads(os.cpu_count() or 4, "port")
    return pyoracle


@pytest.fixture(scope="session")
def golden():
    def load(name):
        d = np.load(os.path.join(GOLDEN, name + ".npz"), allow_pickle=False)
        return {k: d[k] for k in d.files}
    return load


@pytest.fixture(scope="session")
def golden_grid(po, golden):
    """The oracle grid for a golden grid name, checked against the fixture."""
    cache = {}

    def get(name):
        if name not in cache:
            g = golden(f"qgrid_{name}")
            G = po.Grid(int(g["ncol"]), int(g["nrow"]), *g["region"], float(g["alpha_i_deg"]),
                        float(g["energy_kev"]), tuple(g["dn2"]), backend="port")
            cache[name] = (G, g)
        return cache[name]
    return get


@pytest.fixture(scope="session")
def ctx():
    import hipgisaxs_b200 as hg
    from hipgisaxs_b200 import _capi
    import ctypes as C
    n = C.c_int(0)
    try:
        import torch
        if not torch.cuda.is_available():
            pytest.skip("no CUDA device")
    except ImportError:
        pass
    c = hg.Context(0)
    yield c
    c.close()
