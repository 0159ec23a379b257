"""Python mirror of the hgx C ABI: contexts, device-resident q-grids and the kernels.

Arrays may be numpy arrays (host memory) or torch tensors (host or CUDA memory); complex
arrays are complex128 (interleaved re/im).  Calls with host outputs are synchronous; calls
whose inputs and outputs are all CUDA tensors run asynchronously on the context's stream.
"""
from __future__ import annotations

import ctypes as C
import weakref

import numpy as np

from . import _capi
from ._capi import C64, C128, F32C, F64, check, lib

PRECISION = {"f64": F64, "f32c": F32C}
CTYPE = {"c128": C128, "c64": C64}


def _is_tensor(x):
    return hasattr(x, "data_ptr") and hasattr(x, "is_cuda")


def _in(x, dtype):
    """(pointer, keepalive) for an input array."""
    if x is None:
        return None, None
    if _is_tensor(x):
        if not x.is_contiguous():
            raise ValueError("tensor arguments must be contiguous")
        return x.data_ptr(), x
    a = np.ascontiguousarray(x, dtype=dtype)
    return a.ctypes.data, a


def _is_device(x):
    return _is_tensor(x) and x.is_cuda


class Context:
    """One hgx context (a GPU, a stream, scratch memory).  hgx_create / hgx_destroy."""

    def __init__(self, device: int = 0, stream=None):
        h = C.c_void_p()
        check(lib().hgx_create(int(device), C.byref(h)))
        self._h = h
        self.device = device
        self._children = []  # weak references to grids and batches made on this context
        if stream is not None:
            self.set_stream(stream)

    def _register(self, obj):
        self._children.append(weakref.ref(obj))

    @property
    def handle(self):
        return self._h

    def set_stream(self, stream):
        """stream: a cudaStream_t as int, or a torch.cuda.Stream."""
        s = getattr(stream, "cuda_stream", stream)
        check(lib().hgx_set_stream(self._h, C.c_void_p(int(s) if s else 0)))

    def synchronize(self):
        check(lib().hgx_synchronize(self._h))

    def close(self):
        """Closes the objects made on this context (newest first), then the context."""
        if getattr(self, "_h", None):
            for ref in reversed(self._children):
                obj = ref()
                if obj is not None:
                    obj.close()
            self._children = []
            lib().hgx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class QGrid:
    """A device-resident q-grid (replaces the reference's QGrid singleton + per-call uploads)."""

    def __init__(self, ctx: Context, handle):
        self.ctx = ctx
        self._h = handle
        ctx._register(self)
        a = [C.c_int() for _ in range(5)]
        check(lib().hgx_qgrid_info(self._h, *[C.byref(x) for x in a]))
        self.nqy, self.nqz, self.nrow, self.ncol, self.mode = (x.value for x in a)

    @classmethod
    def from_arrays(cls, ctx: Context, qx, qy, qz, ncol: int = 0):
        px, kx = _in(qx, np.float64)
        py, ky = _in(qy, np.float64)
        pz, kz = _in(qz, np.complex128)
        nqy = int(kx.numel() if _is_tensor(kx) else kx.size)
        nqz = int(kz.numel() if _is_tensor(kz) else kz.size)
        h = C.c_void_p()
        check(lib().hgx_qgrid_from_arrays(ctx.handle, nqy, px, py, nqz, pz, int(ncol),
                                          C.byref(h)))
        return cls(ctx, h)

    @classmethod
    def create(cls, ctx: Context, ncol, nrow, qmin_y, qmin_z, qmax_y, qmax_z, alpha_i, k0,
               dn2=(0.0, 0.0)):
        """QGrid::create + create_qz_extended on the device (alpha_i in radians)."""
        h = C.c_void_p()
        check(lib().hgx_qgrid_create(ctx.handle, int(ncol), int(nrow), float(qmin_y),
                                     float(qmin_z), float(qmax_y), float(qmax_z),
                                     float(alpha_i), float(k0), float(dn2[0]), float(dn2[1]),
                                     C.byref(h)))
        return cls(ctx, h)

    @property
    def handle(self):
        return self._h

    def read(self, qz_det=True, alpha=True):
        qx = np.zeros(self.nqy)
        qy = np.zeros(self.nqy)
        qz = np.zeros(self.nqy) if qz_det else None
        al = np.zeros(self.nrow) if alpha else None
        ext = np.zeros(self.nqz, dtype=np.complex128)
        check(lib().hgx_qgrid_read(self.ctx.handle, self._h, qx.ctypes.data, qy.ctypes.data,
                                   None if qz is None else qz.ctypes.data,
                                   None if al is None else al.ctypes.data, ext.ctypes.data))
        return dict(qx=qx, qy=qy, qz=qz, alpha=al, qz_ext=ext)

    def close(self):
        if getattr(self, "_h", None):
            lib().hgx_qgrid_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _rot_arg(rot):
    r = np.ascontiguousarray(np.eye(3) if rot is None else rot, dtype=np.float64).reshape(9)
    return r


def ff_triangles(ctx: Context, grid: QGrid, shape_def, rot=None, precision="f32c", out=None,
                 out_type="c128", pixels_per_thread=0):
    """Numeric form factor of a triangle mesh on `grid` (hgx_ff_triangles_q).

    shape_def: (T, 8) float64 rows (s, nx, ny, nz, cx, cy, cz, pad).  Returns `out` (a
    numpy complex array when not given)."""
    psd, ksd = _in(shape_def, np.float64)
    ntri = int((ksd.numel() if _is_tensor(ksd) else ksd.size) // 8)
    r = _rot_arg(rot)
    ct = CTYPE[out_type]
    if out is None:
        out = np.zeros(grid.nqz, dtype=np.complex64 if ct == C64 else np.complex128)
    pout = out.data_ptr() if _is_tensor(out) else out.ctypes.data
    check(lib().hgx_ff_triangles_q_ex(ctx.handle, grid.handle, psd, ntri, r.ctypes.data,
                                      PRECISION[precision], pout, ct, int(pixels_per_thread)))
    return out


def ff_exact_triangles(ctx: Context, grid: QGrid, tris, rot=None, out=None, out_type="c128"):
    """Exact (polyhedral) triangle form factor on `grid` (hgx_ff_exact_triangles_q), FP64.

    tris: (T, 9) float64 vertex triples (v1, v2, v3).  Returns `out`."""
    pt, kt = _in(tris, np.float64)
    ntri = int((kt.numel() if _is_tensor(kt) else kt.size) // 9)
    r = _rot_arg(rot)
    ct = CTYPE[out_type]
    if out is None:
        out = np.zeros(grid.nqz, dtype=np.complex64 if ct == C64 else np.complex128)
    pout = out.data_ptr() if _is_tensor(out) else out.ctypes.data
    check(lib().hgx_ff_exact_triangles_q(ctx.handle, grid.handle, pt, ntri, r.ctypes.data, pout, ct))
    return out


TUNE_CANDIDATES = (4, 2, 1, -2, -4, -8)


def ff_tune(ctx: Context, grid: QGrid, shape_def, rot=None, out_type="c64", reps=2):
    """Autotune the FP32C kernel's launch shape on `grid` (hgx_ff_tune); later automatic
    calls on this grid use the choice.  Returns (pixels_per_thread, ms, {candidate: ms})."""
    psd, ksd = _in(shape_def, np.float64)
    ntri = int((ksd.numel() if _is_tensor(ksd) else ksd.size) // 8)
    r = _rot_arg(rot)
    best, ms = C.c_int(), C.c_double()
    times = np.zeros(len(TUNE_CANDIDATES))
    check(lib().hgx_ff_tune(ctx.handle, grid.handle, psd, ntri, r.ctypes.data, CTYPE[out_type],
                            int(reps), C.byref(best), C.byref(ms), times.ctypes.data))
    return best.value, ms.value, {p: t for p, t in zip(TUNE_CANDIDATES, times) if t > 0}


def measure_peaks(ctx: Context, sustained_ms: int = 0):
    """(FP32 TFLOP/s, SFU Gop/s) measured by the library's probe kernels."""
    f = C.c_double()
    s = C.c_double()
    check(lib().hgx_measure_peaks(ctx.handle, int(sustained_ms), C.byref(f), C.byref(s)))
    return f.value, s.value


def measure_peak_fp64(ctx: Context):
    """FP64 FMA TFLOP/s measured by the library's DFMA probe."""
    f = C.c_double()
    check(lib().hgx_measure_peak_fp64(ctx.handle, C.byref(f)))
    return f.value


def ff_triangles_arrays(ctx: Context, shape_def, qx, qy, qz, rot=None, precision="f64",
                        out=None):
    """The reference-shaped call (hgx_ff_triangles): explicit arrays, complex128 result
    (written to `out` when given, e.g. a pinned host buffer)."""
    psd, ksd = _in(shape_def, np.float64)
    ntri = int((ksd.numel() if _is_tensor(ksd) else ksd.size) // 8)
    px, kx = _in(qx, np.float64)
    py, ky = _in(qy, np.float64)
    pz, kz = _in(qz, np.complex128)
    r = _rot_arg(rot)
    if out is None:
        out = np.zeros(kz.numel() if _is_tensor(kz) else kz.size, dtype=np.complex128)
    pout = out.data_ptr() if _is_tensor(out) else out.ctypes.data
    nqy = int(kx.numel() if _is_tensor(kx) else kx.size)
    nqz = int(kz.numel() if _is_tensor(kz) else kz.size)
    check(lib().hgx_ff_triangles(ctx.handle, psd, ntri, nqy, px, py, nqz, pz,
                                 r.ctypes.data, PRECISION[precision], pout))
    return out
