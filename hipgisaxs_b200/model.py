"""Python mirror of the C ABI for the analytic form factors, the lattice structure factor,
the DWBA terms and the distance measures (see include/hgx.h for the reference interfaces
each call replaces)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._capi import C64, C128, check, lib
from .core import CTYPE, PRECISION, Context, QGrid, _in, _is_tensor

SHAPE = {"box": 2, "cube": 3, "cylinder": 4, "sphere": 5, "prism3": 8, "prism6": 9,
         "pyramid": 14}
PARAM = {"radius": 2, "xsize": 3, "ysize": 4, "height": 5, "edge": 6, "baseangle": 7}
STAT = {"null": 0, "none": 2, "gaussian": 4, "uniform": 8}
LATTICE = {"bcc": 2, "cubic": 3, "fcc": 4, "fco": 5, "hcp": 6, "hex": 7}


def _ptr(x):
    if x is None:
        return None
    return x.data_ptr() if _is_tensor(x) else x.ctypes.data


def _out(out, n, out_type):
    if out is None:
        out = np.zeros(n, dtype=np.complex64 if CTYPE[out_type] == C64 else np.complex128)
    return out


def param_distribution(stat, pmin, pmax, mean, dev, nvalues):
    cap = 4 * int(nvalues) + 16
    v = np.zeros(cap)
    w = np.zeros(cap)
    n = C.c_int()
    check(lib().hgx_param_distribution(STAT[stat], float(pmin), float(pmax), float(mean),
                                       float(dev), int(nvalues), v.ctypes.data, w.ctypes.data,
                                       cap, C.byref(n)))
    return v[:n.value].copy(), w[:n.value].copy()


def ff_analytic(ctx: Context, grid: QGrid, shape, dims, tau=0.0, eta=0.0, transvec=(0, 0, 0),
                rot=None, out=None, out_type="c128", precision="f64"):
    """dims: up to four (values, weights-or-None) pairs in the order of hgx_ff_analytic;
    precision "f32c" on real-qz grids for cylinders, spheres and boxes."""
    args = []
    keep = []
    for i in range(4):
        if i < len(dims) and dims[i] is not None and len(dims[i][0]):
            v = np.ascontiguousarray(dims[i][0], dtype=np.float64)
            w = None if dims[i][1] is None else np.ascontiguousarray(dims[i][1], dtype=np.float64)
            keep += [v, w]
            args += [len(v), v.ctypes.data, None if w is None else w.ctypes.data]
        else:
            args += [0, None, None]
    tv = np.ascontiguousarray(transvec, dtype=np.float64)
    r = None if rot is None else np.ascontiguousarray(rot, dtype=np.float64).reshape(9)
    out = _out(out, grid.nqz, out_type)
    check(lib().hgx_ff_analytic_ex(ctx.handle, grid.handle, SHAPE[shape], *args, float(tau),
                                   float(eta), tv.ctypes.data, None if r is None else r.ctypes.data,
                                   _ptr(out), CTYPE[out_type], PRECISION[precision]))
    return out


def param_rows(params):
    rows = [[PARAM[p["type"]], STAT[p.get("stat", "none")], p.get("min", 0.0), p.get("max", 0.0),
             p.get("mean", float("nan")), p.get("deviation", 0.0), p.get("nvalues", 1)]
            for p in params]
    return np.ascontiguousarray(np.array(rows, dtype=np.float64).reshape(-1, 7))


def ff_analytic_params(ctx: Context, grid: QGrid, shape, params, tau=0.0, eta=0.0,
                       transvec=(0, 0, 0), rot=None, out=None, out_type="c128", precision="f64"):
    """params: dicts {type, stat, min, max, mean, deviation, nvalues} (HiG shape parameters)."""
    P = params if isinstance(params, np.ndarray) else param_rows(params)
    P = np.ascontiguousarray(P, dtype=np.float64)
    tv = np.ascontiguousarray(transvec, dtype=np.float64)
    r = None if rot is None else np.ascontiguousarray(rot, dtype=np.float64).reshape(9)
    out = _out(out, grid.nqz, out_type)
    check(lib().hgx_ff_analytic_params_ex(ctx.handle, grid.handle, SHAPE[shape], len(P),
                                          P.ctypes.data, float(tau), float(eta), tv.ctypes.data,
                                          None if r is None else r.ctypes.data, _ptr(out),
                                          CTYPE[out_type], PRECISION[precision]))
    return out


def lattice_vectors(kind, hkl="100"):
    abc = np.zeros(9)
    t = np.zeros(3)
    check(lib().hgx_lattice_vectors(LATTICE[kind], hkl.encode(), abc.ctypes.data, t.ctypes.data))
    return abc.reshape(3, 3), t


def sf_lattice(ctx: Context, grid: QGrid, abc, repet, scaling, center=(0, 0, 0), rot=None,
               out=None, out_type="c128", precision="f64"):
    abc9 = np.ascontiguousarray(np.asarray(abc, dtype=np.float64).reshape(9))
    rp = np.ascontiguousarray(repet, dtype=np.float64)
    sc = np.ascontiguousarray(scaling, dtype=np.float64)
    ce = np.ascontiguousarray(center, dtype=np.float64)
    r = None if rot is None else np.ascontiguousarray(rot, dtype=np.float64).reshape(9)
    out = _out(out, grid.nqz, out_type)
    check(lib().hgx_sf_lattice_ex(ctx.handle, grid.handle, abc9.ctypes.data, rp.ctypes.data,
                                  sc.ctypes.data, ce.ctypes.data, None if r is None else r.ctypes.data,
                                  _ptr(out), CTYPE[out_type], PRECISION[precision]))
    return out


def dwba_mesh_grains(ctx: Context, grid: QGrid, shape_def, rots, centers, weights, abc, repet,
                     scaling, fc, dn2, precision="f32c"):
    """The grain loop of one structure (hgx_dwba_mesh_grains): sum over grains of
    |w dn2 sum_k fc_k sf_k ff_k|^2 with each grain's rotation and unit-cell centre."""
    from ._capi import F32C, F64
    psd, ksd = _in(shape_def, np.float64)
    ntri = int((ksd.numel() if _is_tensor(ksd) else ksd.size) // 8)
    r = np.ascontiguousarray(np.asarray(rots, dtype=np.float64).reshape(-1, 9))
    c = np.ascontiguousarray(np.asarray(centers, dtype=np.float64).reshape(-1, 3))
    w = np.ascontiguousarray(np.asarray(weights, dtype=np.float64).reshape(-1))
    if not (len(r) == len(c) == len(w)):
        raise ValueError("one rotation, centre and weight per grain")
    abc9 = np.ascontiguousarray(np.asarray(abc, dtype=np.float64).reshape(9))
    rp = np.ascontiguousarray(repet, dtype=np.float64)
    sc = np.ascontiguousarray(scaling, dtype=np.float64)
    pfc, kfc = _in(fc, np.complex128)
    out = np.zeros(grid.nqy)
    check(lib().hgx_dwba_mesh_grains(ctx.handle, grid.handle, psd, ntri, len(r), r.ctypes.data,
                                     c.ctypes.data, w.ctypes.data, abc9.ctypes.data, rp.ctypes.data,
                                     sc.ctypes.data, pfc, float(dn2[0]), float(dn2[1]),
                                     F64 if precision == "f64" else F32C, out.ctypes.data))
    return out


def dwba_analytic_grains(ctx: Context, grid: QGrid, shape, params, rots, centers, weights, abc,
                         repet, scaling, fc, dn2, tau=0.0, eta=0.0, transvec=(0, 0, 0)):
    """The grain loop of one structure of analytic particles (hgx_dwba_analytic_grains)."""
    P = params if isinstance(params, np.ndarray) else param_rows(params)
    P = np.ascontiguousarray(P, dtype=np.float64)
    tv = np.ascontiguousarray(transvec, dtype=np.float64)
    r = np.ascontiguousarray(np.asarray(rots, dtype=np.float64).reshape(-1, 9))
    c = np.ascontiguousarray(np.asarray(centers, dtype=np.float64).reshape(-1, 3))
    w = np.ascontiguousarray(np.asarray(weights, dtype=np.float64).reshape(-1))
    if not (len(r) == len(c) == len(w)):
        raise ValueError("one rotation, centre and weight per grain")
    abc9 = np.ascontiguousarray(np.asarray(abc, dtype=np.float64).reshape(9))
    rp = np.ascontiguousarray(repet, dtype=np.float64)
    sc = np.ascontiguousarray(scaling, dtype=np.float64)
    pfc, kfc = _in(fc, np.complex128)
    out = np.zeros(grid.nqy)
    check(lib().hgx_dwba_analytic_grains(ctx.handle, grid.handle, SHAPE[shape], len(P), P.ctypes.data,
                                         float(tau), float(eta), tv.ctypes.data, len(r),
                                         r.ctypes.data, c.ctypes.data, w.ctypes.data,
                                         abc9.ctypes.data, rp.ctypes.data, sc.ctypes.data, pfc,
                                         float(dn2[0]), float(dn2[1]), out.ctypes.data))
    return out


def save_gisaxs(path, image, ctx: Context = None):
    """Writes a (nrow, ncol) image as the reference's ".out" text (hgx_save_gisaxs)."""
    if _is_tensor(image):
        nrow, ncol = image.shape
        ptr, keep = image.data_ptr(), image
    else:
        keep = np.ascontiguousarray(image, dtype=np.float64)
        nrow, ncol = keep.shape
        ptr = keep.ctypes.data
    check(lib().hgx_save_gisaxs(None if ctx is None else ctx.handle, ptr, int(nrow), int(ncol),
                                str(path).encode()))


def structure_sum(ctx: Context, intensities, iratios):
    """Sum over structures weighted by their (rescaled) iratios (hgx_structure_sum)."""
    I = np.ascontiguousarray(intensities, dtype=np.float64)
    I2 = I.reshape(len(I), -1)
    r = np.ascontiguousarray(iratios, dtype=np.float64)
    out = np.zeros(I2.shape[1])
    check(lib().hgx_structure_sum(ctx.handle, len(I2), I2.shape[1], I2.ctypes.data, r.ctypes.data,
                                  out.ctypes.data))
    return out.reshape(I.shape[1:])


def gaussian_smearing(ctx: Context, image, sigma):
    """Gaussian smearing of a (nrow, ncol) image (hgx_gaussian_smearing); returns a smeared
    copy of a numpy image, or smears a contiguous device tensor in place and returns it."""
    if _is_tensor(image):
        nrow, ncol = image.shape
        check(lib().hgx_gaussian_smearing(ctx.handle, image.data_ptr(), int(ncol), int(nrow),
                                          float(sigma)))
        return image
    img = np.ascontiguousarray(image, dtype=np.float64).copy()
    nrow, ncol = img.shape
    check(lib().hgx_gaussian_smearing(ctx.handle, img.ctypes.data, int(ncol), int(nrow),
                                      float(sigma)))
    return img


def normalize(ctx: Context, data):
    """HipGISAXS::normalize of a copy of `data` (hgx_normalize): (normalised, flag)."""
    d = np.ascontiguousarray(data, dtype=np.float64).copy()
    ok = C.c_int()
    check(lib().hgx_normalize(ctx.handle, d.ctypes.data, d.size, C.byref(ok)))
    return d, bool(ok.value)


def sf_paracrystal(ctx: Context, grid: QGrid, dims, lattice="cubic", dist=(0.0, 0.0),
                   sdev=(0.0, 0.0), domain=1.0, out=None, out_type="c128"):
    """Paracrystal structure factor (hgx_sf_paracrystal): dims 1, or 2 on a cubic or hex
    lattice; dist = (x, y) mean distances, sdev = (x, y) standard deviations."""
    out = _out(out, grid.nqz, out_type)
    check(lib().hgx_sf_paracrystal(ctx.handle, grid.handle, int(dims), LATTICE[lattice],
                                   float(dist[0]), float(dist[1]), float(sdev[0]), float(sdev[1]),
                                   float(domain), _ptr(out), CTYPE[out_type]))
    return out


def sf_percus_yevick(ctx: Context, grid: QGrid, diameter, volfract, dims=2, out=None,
                     out_type="c128"):
    """Percus-Yevick hard-sphere structure factor (hgx_sf_percus_yevick), dims 2 or 3."""
    out = _out(out, grid.nqz, out_type)
    check(lib().hgx_sf_percus_yevick(ctx.handle, grid.handle, float(diameter), float(volfract),
                                     int(dims), _ptr(out), CTYPE[out_type]))
    return out


def propagation_coeffs(ctx: Context, grid: QGrid, layers, k0, alpha_i, particle_order=0,
                       alpha=None, per_row=False, out=None):
    """layers: (delta, beta, thickness, order) tuples, order -1 = substrate."""
    d = np.ascontiguousarray([l[0] for l in layers], dtype=np.float64)
    b = np.ascontiguousarray([l[1] for l in layers], dtype=np.float64)
    t = np.ascontiguousarray([l[2] for l in layers], dtype=np.float64)
    o = np.ascontiguousarray([int(l[3]) for l in layers], dtype=np.int32)
    n = 4 * (grid.nrow if per_row else grid.nrow * grid.ncol)
    if out is None:
        out = np.zeros(n, dtype=np.complex128)
    pa, ka = _in(alpha, np.float64)
    check(lib().hgx_propagation_coeffs(ctx.handle, grid.handle, len(layers), d.ctypes.data,
                                       b.ctypes.data, t.ctypes.data, o.ctypes.data, float(k0),
                                       float(alpha_i), int(particle_order), pa, _ptr(out),
                                       1 if per_row else 0))
    return out


def dwba_combine(ctx: Context, fc, sf, ff, weight=1.0, intensity=None):
    """intensity += |w sum_k fc sf ff|^2 (fc None: SAXS branch).  Returns intensity."""
    nb = ff.numel() if _is_tensor(ff) else len(ff)
    n = nb // 4 if fc is not None else nb
    if intensity is None:
        intensity = np.zeros(n)
    pfc, kfc = _in(fc, np.complex128)
    psf, ksf = _in(sf, np.complex128)
    if _is_tensor(ff):
        ftype = C64 if str(ff.dtype) == "torch.complex64" else C128
        pff = ff.data_ptr()
    else:
        ftype = C64 if ff.dtype == np.complex64 else C128
        ff = np.ascontiguousarray(ff)
        pff = ff.ctypes.data
    check(lib().hgx_dwba_combine(ctx.handle, n, pfc, psf, pff, ftype, float(weight),
                                 _ptr(intensity)))
    return intensity


def _scalar(fn, ctx, *arrays, extra=()):
    ptrs = []
    keep = []
    n = None
    for a, dt in arrays:
        p, k = _in(a, dt)
        ptrs.append(p)
        keep.append(k)
        if k is not None and n is None:
            n = k.numel() if _is_tensor(k) else k.size
    out = np.zeros(1)
    check(fn(ctx.handle, int(n), *ptrs, *extra, out.ctypes.data))
    return float(out[0])


def chi2(ctx: Context, model, counts, mask=None, scale=1.0):
    p1, k1 = _in(model, np.float64)
    p2, k2 = _in(counts, np.float64)
    p3, k3 = _in(mask, np.uint32)
    n = k1.numel() if _is_tensor(k1) else k1.size
    out = np.zeros(1)
    check(lib().hgx_chi2(ctx.handle, int(n), p1, p2, p3, float(scale), out.ctypes.data))
    return float(out[0])


def abs_diff_square(ctx: Context, ref, data, mask):
    p1, k1 = _in(ref, np.float64)
    p2, k2 = _in(data, np.float64)
    p3, k3 = _in(mask, np.uint32)
    n = k1.numel() if _is_tensor(k1) else k1.size
    out = np.zeros(1)
    check(lib().hgx_abs_diff_square(ctx.handle, int(n), p1, p2, p3, out.ctypes.data))
    return float(out[0])


def residual_vector(ctx: Context, ref, data, mask=None):
    p1, k1 = _in(ref, np.float64)
    p2, k2 = _in(data, np.float64)
    p3, k3 = _in(mask, np.uint32)
    n = k1.numel() if _is_tensor(k1) else k1.size
    out = np.zeros(n)
    check(lib().hgx_residual_vector(ctx.handle, int(n), p1, p2, p3, out.ctypes.data))
    return out
