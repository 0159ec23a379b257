"""hipgisaxs_b200 — a B200-native (sm_100a) GISAXS forward model.

The hot path of the reference simulator (tacaswell/hipgisaxs) — the triangulated-mesh
form factor, the analytic form factors, the lattice structure factor and the four-term
DWBA combination — as hand-written CUDA kernels behind a C ABI (include/hgx.h,
libhgx.so).  This Python package is a thin host-side mirror of that ABI; the C++ drop-in
classes with the reference's signatures are declared in include/hgx_hig.hpp and implemented
in csrc/hig_dropin.cpp.
"""
from ._capi import HgxError, lib  # noqa: F401
from .core import (Context, QGrid, ff_exact_triangles, ff_triangles,  # noqa: F401
                   ff_triangles_arrays, ff_tune, measure_peak_fp64, measure_peaks)

__all__ = ["Context", "QGrid", "ff_triangles", "ff_triangles_arrays", "ff_exact_triangles",
           "ff_tune", "HgxError", "lib"]
