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
