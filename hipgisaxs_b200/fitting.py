"""Python mirror of the fitting entry points: the fused cylinder-lattice model with its
chi^2 and adjoint gradient, batched over candidates (hgx_cyl_batch_*), plus the
finite-difference gradient of the plain FP64 form (the reference fitter's method)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._capi import F32C, F64, check, lib
from .core import PRECISION, Context, QGrid, _in

MODEL_LEN = 16
THETA = ("radius", "height", "lattice_a", "phi")


def model_block(radius, height, lattice_a, phi=0.0, spread=0.0, nsamples=1, repet=(20, 20, 1),
                dn2=(0.0, 0.0), center=(0.0, 0.0, 0.0), weight=1.0, smooth_sampling=False):
    """The 16-double model block of hgx_cyl_batch_* (see include/hgx.h)."""
    m = np.zeros(MODEL_LEN)
    m[15] = 1.0 if smooth_sampling else 0.0
    m[0], m[1], m[2], m[3] = radius, height, lattice_a, phi
    m[4], m[5] = spread, nsamples
    m[6:9] = repet
    m[9:11] = dn2
    m[11:14] = center
    m[14] = weight
    return m


def mesh_to_shape_def(ctx: Context, verts, faces):
    """Triangle tuples (s, n, c) of a mesh on the device, one row per face (degenerate faces
    get s = 0)."""
    v = np.ascontiguousarray(verts, dtype=np.float64).reshape(-1, 3)
    f = np.ascontiguousarray(faces, dtype=np.int32).reshape(-1, 3)
    out = np.zeros((len(f), 8))
    check(lib().hgx_mesh_to_shape_def(ctx.handle, len(v), v.ctypes.data, len(f), f.ctypes.data,
                                      out.ctypes.data))
    return out


def mesh_chi2_grad(ctx: Context, grid: QGrid, verts, faces, rowfc, dn2, counts=None, mask=None,
                   scale=1.0, weight=1.0, rot=None, want_grad=True, want_intensity=False,
                   precision="f32c"):
    """(chi2, grad[nv, 3] or None, intensity[N] or None) for a mesh in DWBA; precision "f32c"
    (FP32C forward and backward) or "f64" (plain FP64 throughout)."""
    v = np.ascontiguousarray(verts, dtype=np.float64).reshape(-1, 3)
    f = np.ascontiguousarray(faces, dtype=np.int32).reshape(-1, 3)
    rf = np.ascontiguousarray(rowfc, dtype=np.complex128)
    r = None if rot is None else np.ascontiguousarray(rot, dtype=np.float64).reshape(9)
    pc, cnt = _in(counts, np.float64)  # host arrays or device tensors
    pm, mk = _in(mask, np.uint32)
    chi = C.c_double()
    gv = np.zeros((len(v), 3)) if want_grad else None
    inten = np.zeros(grid.nrow * grid.ncol) if want_intensity else None
    check(lib().hgx_mesh_chi2_grad_ex(
        ctx.handle, grid.handle, len(v), v.ctypes.data, len(f), f.ctypes.data,
        None if r is None else r.ctypes.data, rf.ctypes.data, float(dn2[0]), float(dn2[1]),
        float(weight), pc, pm, float(scale), C.byref(chi),
        None if gv is None else gv.ctypes.data, None if inten is None else inten.ctypes.data,
        PRECISION[precision]))
    return chi.value, gv, inten


class CylinderBatch:
    """hgx_cyl_batch: candidates with ROIs on one device grid."""

    def __init__(self, ctx: Context, grid: QGrid, rowfc, abc, rois, counts=None, mask=None,
                 scale=1.0, precision="f32c"):
        self.ctx, self.grid = ctx, grid
        rf = np.ascontiguousarray(rowfc, dtype=np.complex128)
        abc9 = np.ascontiguousarray(np.asarray(abc, dtype=np.float64).reshape(9))
        r = np.ascontiguousarray(np.asarray(rois, dtype=np.int32).reshape(-1, 4))
        self.rois = r
        self.ncand = len(r)
        cnt = None if counts is None else np.ascontiguousarray(counts, dtype=np.float64)
        mk = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint32)
        h = C.c_void_p()
        check(lib().hgx_cyl_batch_create(ctx.handle, grid.handle, rf.ctypes.data, abc9.ctypes.data,
                                         self.ncand, r.ctypes.data,
                                         None if cnt is None else cnt.ctypes.data,
                                         None if mk is None else mk.ctypes.data, float(scale),
                                         F64 if precision == "f64" else F32C, C.byref(h)))
        self._h = h
        ctx._register(self)
        n1, n2 = C.c_long(), C.c_long()
        check(lib().hgx_cyl_batch_info(h, C.byref(n1), C.byref(n2)))
        self.npx = n1.value
        self.offsets = np.concatenate([[0], np.cumsum(r[:, 2].astype(np.int64) * r[:, 3])])

    @property
    def nitems(self):
        """Work items of the current tile shape."""
        n1, n2 = C.c_long(), C.c_long()
        check(lib().hgx_cyl_batch_info(self._h, C.byref(n1), C.byref(n2)))
        return n2.value

    @staticmethod
    def shapes():
        """The tile-shape table: [(threads per block, pixels per thread), ...]."""
        out, k = [], 0
        while True:
            t, p = C.c_int(), C.c_int()
            if lib().hgx_cyl_shape_info(k, C.byref(t), C.byref(p)) != 0:
                return out
            out.append((t.value, p.value))
            k += 1

    @property
    def shape(self):
        s = C.c_int()
        check(lib().hgx_cyl_batch_get_shape(self._h, C.byref(s)))
        return s.value

    @shape.setter
    def shape(self, k):
        check(lib().hgx_cyl_batch_set_shape(self._h, int(k)))

    def tune(self, models, reps=3):
        """Autotune the tile shape on this batch: (best shape, its ms, ms of every shape)."""
        m = self._models(models)
        best, ms = C.c_int(), C.c_double()
        times = np.zeros(len(self.shapes()))
        check(lib().hgx_cyl_batch_tune(self._h, m.ctypes.data, int(reps), C.byref(best),
                                       C.byref(ms), times.ctypes.data))
        return best.value, ms.value, times

    def _models(self, models):
        m = np.ascontiguousarray(np.asarray(models, dtype=np.float64).reshape(-1, MODEL_LEN))
        if len(m) != self.ncand:
            raise ValueError("one model block per candidate")
        return m

    def eval(self, models):
        """(chi2[ncand], grad[ncand, 4]) for theta = (R, H, a, phi)."""
        m = self._models(models)
        out = np.zeros((self.ncand, 5))
        check(lib().hgx_cyl_batch_eval(self._h, m.ctypes.data, out.ctypes.data))
        return out[:, 0].copy(), out[:, 1:].copy()

    def forward(self, models):
        m = self._models(models)
        out = np.zeros(self.npx)
        check(lib().hgx_cyl_batch_forward(self._h, m.ctypes.data, out.ctypes.data))
        return [out[self.offsets[i]:self.offsets[i + 1]].reshape(self.rois[i, 2], self.rois[i, 3])
                for i in range(self.ncand)]

    def plain_forward(self, cand, model):
        m = np.ascontiguousarray(model, dtype=np.float64)
        n = int(self.rois[cand, 2]) * int(self.rois[cand, 3])
        out = np.zeros(n)
        check(lib().hgx_cyl_plain_forward(self._h, int(cand), m.ctypes.data, out.ctypes.data))
        return out

    def close(self):
        if getattr(self, "_h", None):
            lib().hgx_cyl_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
