"""TEST INFRASTRUCTURE — Python access to the CPU oracle.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU legs import this module, and
only as the checker.  Two backends with one API:

* ``"port"``: ``oracle/liboracle.so``, the plain-C FP64 restatement (hgx_oracle.c);
* ``"ref"``:  ``oracle/_ref/libhigref.so``, the reference's own CPU sources compiled by
  ``make -C oracle ref`` (present only where the reference tree was available to build it).

Complex arrays are numpy complex128.  Grids follow the reference's layout: N = nrow*ncol
pixels flattened row-major, extended (DWBA) arrays hold 4 blocks of N.
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libhigref.so")

# enums of include/common/enums.hpp (reference)
SHAPE = {"box": 2, "cube": 3, "cylinder": 4, "sphere": 5, "prism3": 8, "prism6": 9,
         "pyramid": 14}
PARAM = {"radius": 2, "xsize": 3, "ysize": 4, "height": 5, "edge": 6, "baseangle": 7}
STAT = {"null": 0, "none": 2, "gaussian": 4, "uniform": 8}
LATTICE = {"bcc": 2, "cubic": 3, "fcc": 4, "fco": 5, "hcp": 6, "hex": 7}

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_up = C.POINTER(C.c_uint)


def _p(a):
    return a.ctypes.data_as(_dp)


def _cbuf(a):
    a = np.ascontiguousarray(a, dtype=np.complex128)
    return a, a.view(np.float64)


_libs: dict = {}


def available(backend: str) -> bool:
    return os.path.exists(PORT_SO if backend == "port" else REF_SO)


def lib(backend: str = "port"):
    if backend in _libs:
        return _libs[backend]
    path = PORT_SO if backend == "port" else REF_SO
    if not os.path.exists(path):
        raise FileNotFoundError(f"oracle library missing: {path} (run `make -C oracle`"
                                f"{' ref' if backend == 'ref' else ''})")
    L = C.CDLL(path)
    _libs[backend] = L
    return L


def set_threads(n: int, backend: str = "port") -> int:
    L = lib(backend)
    f = L.orc_set_threads if backend == "port" else L.ref_set_threads
    f.restype = C.c_int
    return f(C.c_int(n))


def k0_from_kev(energy_kev: float) -> float:
    """HipGISAXS::init, src/sim/hipgisaxs_main.cpp:144-158: lambda = 1.23984/E, k0 = 2pi/lambda."""
    lam = 1.23984 / energy_kev
    return 2 * 3.141592653589793 / lam


class Grid:
    """A detector q-grid (QGrid::create) plus the DWBA extended qz for a particle layer."""

    _current_ref = None  # the reference keeps one QGrid singleton

    def __init__(self, ncol, nrow, qmin_y, qmin_z, qmax_y, qmax_z, alpha_i_deg, energy_kev,
                 dn2=(0.0, 0.0), backend="port"):
        self.ncol, self.nrow = int(ncol), int(nrow)
        self.n = self.ncol * self.nrow
        self.region = (qmin_y, qmin_z, qmax_y, qmax_z)
        self.alpha_i = alpha_i_deg * 3.141592653589793 / 180  # PI_ as the reference uses
        self.k0 = k0_from_kev(energy_kev)
        self.dn2 = dn2
        self.backend = backend
        self.qx = np.zeros(self.n)
        self.qy = np.zeros(self.n)
        self.qz = np.zeros(self.n)
        self.alpha = np.zeros(self.nrow)
        self.qz_ext = np.zeros(4 * self.n, dtype=np.complex128)
        self._build()

    def _build(self):
        L = lib(self.backend)
        a = (C.c_double(self.region[0]), C.c_double(self.region[1]), C.c_double(self.region[2]),
             C.c_double(self.region[3]), C.c_double(self.alpha_i), C.c_double(self.k0))
        if self.backend == "port":
            rc = L.orc_qgrid_create(C.c_int(self.ncol), C.c_int(self.nrow), *a, _p(self.qx),
                                    _p(self.qy), _p(self.qz), _p(self.alpha))
            assert rc == 0, rc
            ext = self.qz_ext.view(np.float64)
            rc = L.orc_qz_extended(C.c_int(self.n), _p(self.qz), C.c_double(self.k0),
                                   C.c_double(self.alpha_i), C.c_double(self.dn2[0]),
                                   C.c_double(self.dn2[1]), _p(ext))
            assert rc == 0, rc
        else:
            self.activate()

    def reextend(self, alpha_i_deg):
        """create_qz_extended for another incidence angle over this detector grid (the
        reference's scans keep the grid of the first angle); later calls that take the grid's
        alpha_i (propagation_coeffs) use the new one."""
        assert self.backend == "port"
        self.alpha_i = alpha_i_deg * 3.141592653589793 / 180
        rc = lib("port").orc_qz_extended(C.c_int(self.n), _p(self.qz), C.c_double(self.k0),
                                         C.c_double(self.alpha_i), C.c_double(self.dn2[0]),
                                         C.c_double(self.dn2[1]), _p(self.qz_ext.view(np.float64)))
        assert rc == 0, rc

    def activate(self):
        """Make this grid the reference's QGrid singleton (ref backend only)."""
        if self.backend != "ref":
            return
        if Grid._current_ref is self:
            return
        L = lib("ref")
        a = (C.c_double(self.region[0]), C.c_double(self.region[1]), C.c_double(self.region[2]),
             C.c_double(self.region[3]), C.c_double(self.alpha_i), C.c_double(self.k0))
        rc = L.ref_qgrid_create(C.c_int(self.ncol), C.c_int(self.nrow), *a, _p(self.qx),
                                _p(self.qy), _p(self.qz), _p(self.alpha))
        assert rc == 0, rc
        ext = self.qz_ext.view(np.float64)
        rc = L.ref_qz_extended(C.c_double(self.k0), C.c_double(self.alpha_i),
                               C.c_double(self.dn2[0]), C.c_double(self.dn2[1]), _p(ext))
        assert rc == 0, rc
        Grid._current_ref = self


def ff_approx_triangle(shape_def, qx, qy, qz, rot=None, backend="port"):
    """NumericFormFactorC::compute_approx_triangle on explicit arrays (qz complex, any length
    that is a multiple of len(qx))."""
    L = lib(backend)
    sd = np.ascontiguousarray(shape_def, dtype=np.float64).reshape(-1, 8)
    qx = np.ascontiguousarray(qx, dtype=np.float64)
    qy = np.ascontiguousarray(qy, dtype=np.float64)
    qz, qzf = _cbuf(qz)
    r = np.ascontiguousarray(np.eye(3) if rot is None else rot, dtype=np.float64).reshape(9)
    out = np.zeros(len(qz), dtype=np.complex128)
    f = L.orc_ff_approx_triangle if backend == "port" else L.ref_ff_approx_triangle
    rc = f(_p(sd), C.c_int(len(sd)), C.c_int(len(qx)), _p(qx), _p(qy), C.c_int(len(qz)),
           _p(qzf), _p(r), _p(out.view(np.float64)))
    if rc <= 0:
        raise RuntimeError(f"ff_approx_triangle failed rc={rc}")
    return out


def ff_exact_triangle(tris, qx, qy, qz, rot=None, backend="port"):
    """NumericFormFactorC::compute_exact_triangle on explicit arrays; tris: (T, 9) vertices
    (v1, v2, v3) of each triangle."""
    L = lib(backend)
    tv = np.ascontiguousarray(tris, dtype=np.float64).reshape(-1, 9)
    qx = np.ascontiguousarray(qx, dtype=np.float64)
    qy = np.ascontiguousarray(qy, dtype=np.float64)
    qz, qzf = _cbuf(qz)
    r = np.ascontiguousarray(np.eye(3) if rot is None else rot, dtype=np.float64).reshape(9)
    out = np.zeros(len(qz), dtype=np.complex128)
    f = L.orc_ff_exact_triangle if backend == "port" else L.ref_ff_exact_triangle
    rc = f(_p(tv), C.c_int(len(tv)), C.c_int(len(qx)), _p(qx), _p(qy), C.c_int(len(qz)),
           _p(qzf), _p(r), _p(out.view(np.float64)))
    if rc <= 0:
        raise RuntimeError(f"ff_exact_triangle failed rc={rc}")
    return out


def mesh_triangles(verts, faces):
    """(T, 9) vertex triples of a mesh, as NumericFormFactor::compute2 builds triangle_t from
    an OBJ mesh (src/ff/ff_num.cpp:66-80)."""
    v = np.asarray(verts, dtype=np.float64).reshape(-1, 3)
    f = np.asarray(faces).reshape(-1, 3)
    return np.ascontiguousarray(v[f].reshape(-1, 9))


def mesh_to_shape_def(verts, faces):
    L = lib("port")
    v = np.ascontiguousarray(verts, dtype=np.float64).reshape(-1, 3)
    f = np.ascontiguousarray(faces, dtype=np.int32).reshape(-1, 3)
    out = np.zeros((len(f), 8))
    t = L.orc_mesh_to_shape_def(C.c_int(len(v)), _p(v), C.c_int(len(f)),
                                f.ctypes.data_as(_ip), _p(out))
    if t < 0:
        raise ValueError("bad face index")
    return out[:t]


def param_rows(params):
    """params: list of dicts {type, stat, min, max, mean, deviation, nvalues} -> (n, 7)."""
    rows = []
    for p in params:
        rows.append([PARAM[p["type"]], STAT[p.get("stat", "none")], p.get("min", 0.0),
                     p.get("max", 0.0), p.get("mean", float("nan")), p.get("deviation", 0.0),
                     p.get("nvalues", 1)])
    return np.ascontiguousarray(np.array(rows, dtype=np.float64).reshape(-1, 7))


def param_distribution(stat, pmin, pmax, mean, dev, nvalues):
    L = lib("port")
    cap = max(16, 4 * int(nvalues) + 8)
    dim = np.zeros(cap)
    w = np.zeros(cap)
    n = L.orc_param_distribution(C.c_int(STAT[stat]), C.c_double(pmin), C.c_double(pmax),
                                 C.c_double(mean), C.c_double(dev), C.c_int(int(nvalues)),
                                 _p(dim), _p(w), C.c_int(cap))
    if n < 0:
        raise ValueError("param_distribution failed")
    return dim[:n].copy(), w[:n].copy()


def ff_analytic(grid: Grid, shape, params, tau=0.0, eta=0.0, transvec=(0, 0, 0), rot=None,
                backend=None):
    backend = backend or grid.backend
    L = lib(backend)
    P = param_rows(params)
    tv = np.ascontiguousarray(transvec, dtype=np.float64)
    r = np.ascontiguousarray(np.eye(3) if rot is None else rot, dtype=np.float64).reshape(9)
    out = np.zeros(4 * grid.n, dtype=np.complex128)
    if backend == "port":
        qz, qzf = _cbuf(grid.qz_ext)
        rc = L.orc_ff_analytic(C.c_int(SHAPE[shape]), C.c_int(len(P)), _p(P), C.c_double(tau),
                               C.c_double(eta), _p(tv), _p(r), C.c_int(grid.n), _p(grid.qx),
                               _p(grid.qy), C.c_int(4 * grid.n), _p(qzf),
                               _p(out.view(np.float64)))
    else:
        grid.activate()
        rc = L.ref_ff_analytic(C.c_int(SHAPE[shape]), C.c_int(len(P)), _p(P), C.c_double(tau),
                               C.c_double(eta), _p(tv), _p(r), _p(out.view(np.float64)))
    if rc <= 0:
        raise RuntimeError(f"ff_analytic({shape}) failed rc={rc}")
    return out


def lattice_vectors(kind, hkl="100"):
    L = lib("port")
    a, b, c, t = (np.zeros(3) for _ in range(4))
    rc = L.orc_lattice_vectors(C.c_int(LATTICE[kind]), C.c_char_p(hkl.encode()), _p(a), _p(b),
                               _p(c), _p(t))
    if rc != 0:
        raise ValueError(f"lattice {kind}/{hkl}")
    return a, b, c, t


def sf_lattice(grid: Grid, abc, repet, scaling, center=(0, 0, 0), rot=None, backend=None):
    backend = backend or grid.backend
    L = lib(backend)
    abc9 = np.ascontiguousarray(np.asarray(abc, dtype=np.float64).reshape(9))
    rp = np.ascontiguousarray(repet, dtype=np.float64)
    sc = np.ascontiguousarray(scaling, dtype=np.float64)
    ce = np.ascontiguousarray(center, dtype=np.float64)
    r = np.ascontiguousarray(np.eye(3) if rot is None else rot, dtype=np.float64).reshape(9)
    out = np.zeros(4 * grid.n, dtype=np.complex128)
    if backend == "port":
        qz, qzf = _cbuf(grid.qz_ext)
        rc = L.orc_sf_lattice(_p(abc9), _p(rp), _p(sc), _p(ce), _p(r), C.c_int(grid.n),
                              _p(grid.qx), _p(grid.qy), C.c_int(4 * grid.n), _p(qzf),
                              _p(out.view(np.float64)))
    else:
        grid.activate()
        rc = L.ref_sf_lattice(_p(abc9), _p(rp), _p(sc), _p(ce), _p(r), C.c_int(1),
                              _p(out.view(np.float64)))
    if rc <= 0:
        raise RuntimeError(f"sf_lattice failed rc={rc}")
    return out


def sf_paracrystal(grid: Grid, dims, lattice, dx, dy, sx, sy, dom, backend=None):
    """StructureFactor paracrystal branch on the grid's extended qz (4N values)."""
    backend = backend or grid.backend
    L = lib(backend)
    out = np.zeros(4 * grid.n, dtype=np.complex128)
    if backend == "port":
        rc = L.orc_sf_paracrystal(C.c_int(dims), C.c_int(lattice), C.c_double(dx), C.c_double(dy),
                                  C.c_double(sx), C.c_double(sy), C.c_double(dom), C.c_int(grid.n),
                                  _p(grid.qx), _p(grid.qy), C.c_int(4 * grid.n),
                                  _p(out.view(np.float64)))
    else:
        grid.activate()
        rc = L.ref_sf_paracrystal(C.c_int(dims), C.c_int(lattice), C.c_double(dx), C.c_double(dy),
                                  C.c_double(sx), C.c_double(sy), C.c_double(dom), C.c_int(1),
                                  _p(out.view(np.float64)))
    if rc <= 0:
        raise RuntimeError(f"sf_paracrystal failed rc={rc}")
    return out


def sf_percus_yevick(grid: Grid, dia, volf, dims, backend=None):
    """StructureFactor Percus-Yevick branch on the grid's extended qz (4N values)."""
    backend = backend or grid.backend
    return (sf_percus_yevick_arrays(dia, volf, dims, grid.qx, grid.qy, grid.qz_ext)
            if backend == "port" else _py_ref(grid, dia, volf, dims))


def _py_ref(grid, dia, volf, dims):
    L = lib("ref")
    out = np.zeros(4 * grid.n, dtype=np.complex128)
    grid.activate()
    rc = L.ref_sf_percus_yevick(C.c_double(dia), C.c_double(volf), C.c_int(dims), C.c_int(1),
                                _p(out.view(np.float64)))
    if rc <= 0:
        raise RuntimeError(f"sf_percus_yevick failed rc={rc}")
    return out


def sf_percus_yevick_arrays(dia, volf, dims, qx, qy, qz):
    """Port backend on explicit arrays (q-point i uses qx/qy[i % len(qx)])."""
    L = lib("port")
    qx = np.ascontiguousarray(qx, dtype=np.float64)
    qy = np.ascontiguousarray(qy, dtype=np.float64)
    qz, qzf = _cbuf(qz)
    out = np.zeros(len(qz), dtype=np.complex128)
    rc = L.orc_sf_percus_yevick(C.c_double(dia), C.c_double(volf), C.c_int(dims), C.c_int(len(qx)),
                                _p(qx), _p(qy), C.c_int(len(qz)), _p(qzf), _p(out.view(np.float64)))
    if rc <= 0:
        raise RuntimeError(f"sf_percus_yevick failed rc={rc}")
    return out


def sf_lattice_arrays(abc, repet, scaling, center, rot, qx, qy, qz):
    """Port backend on explicit arrays (qz complex; q-point i uses qx/qy[i % len(qx)])."""
    L = lib("port")
    abc9 = np.ascontiguousarray(np.asarray(abc, dtype=np.float64).reshape(9))
    rp = np.ascontiguousarray(repet, dtype=np.float64)
    sc = np.ascontiguousarray(scaling, dtype=np.float64)
    ce = np.ascontiguousarray(center, dtype=np.float64)
    r = np.ascontiguousarray(np.eye(3) if rot is None else rot, dtype=np.float64).reshape(9)
    qx = np.ascontiguousarray(qx, dtype=np.float64)
    qy = np.ascontiguousarray(qy, dtype=np.float64)
    qz, qzf = _cbuf(qz)
    out = np.zeros(len(qz), dtype=np.complex128)
    L.orc_sf_lattice(_p(abc9), _p(rp), _p(sc), _p(ce), _p(r), C.c_int(len(qx)), _p(qx), _p(qy),
                     C.c_int(len(qz)), _p(qzf), _p(out.view(np.float64)))
    return out


def ff_analytic_arrays(shape, params, qx, qy, qz, tau=0.0, eta=0.0, transvec=(0, 0, 0),
                       rot=None):
    """Port backend on explicit arrays."""
    L = lib("port")
    P = param_rows(params)
    tv = np.ascontiguousarray(transvec, dtype=np.float64)
    r = np.ascontiguousarray(np.eye(3) if rot is None else rot, dtype=np.float64).reshape(9)
    qx = np.ascontiguousarray(qx, dtype=np.float64)
    qy = np.ascontiguousarray(qy, dtype=np.float64)
    qz, qzf = _cbuf(qz)
    out = np.zeros(len(qz), dtype=np.complex128)
    rc = L.orc_ff_analytic(C.c_int(SHAPE[shape]), C.c_int(len(P)), _p(P), C.c_double(tau),
                           C.c_double(eta), _p(tv), _p(r), C.c_int(len(qx)), _p(qx), _p(qy),
                           C.c_int(len(qz)), _p(qzf), _p(out.view(np.float64)))
    if rc <= 0:
        raise RuntimeError(f"ff_analytic({shape}) failed rc={rc}")
    return out


def propagation_coeffs(grid: Grid, layers, particle_order=0, backend=None):
    """layers: list of (delta, beta, thickness, order); order -1 = substrate."""
    backend = backend or grid.backend
    L = lib(backend)
    d = np.ascontiguousarray([l[0] for l in layers], dtype=np.float64)
    b = np.ascontiguousarray([l[1] for l in layers], dtype=np.float64)
    t = np.ascontiguousarray([l[2] for l in layers], dtype=np.float64)
    o = np.ascontiguousarray([l[3] for l in layers], dtype=np.int32)
    out = np.zeros(4 * grid.n, dtype=np.complex128)
    if backend == "port":
        rc = L.orc_propagation_coeffs(C.c_int(len(layers)), _p(d), _p(b), _p(t),
                                      o.ctypes.data_as(_ip), C.c_double(grid.k0),
                                      C.c_double(grid.alpha_i), C.c_int(particle_order),
                                      C.c_int(grid.nrow), C.c_int(grid.ncol), _p(grid.alpha),
                                      _p(out.view(np.float64)))
        if rc != 0:
            raise RuntimeError(f"propagation_coeffs failed rc={rc}")
    else:
        grid.activate()
        rc = L.ref_propagation_coeffs(C.c_int(len(layers)), _p(d), _p(b), _p(t),
                                      o.ctypes.data_as(_ip), C.c_double(grid.k0),
                                      C.c_double(grid.alpha_i), C.c_int(particle_order),
                                      _p(out.view(np.float64)))
        if rc <= 0:
            raise RuntimeError(f"propagation_coeffs failed rc={rc}")
    return out


def parratt(layers_stack, alpha, k0, order, backend="port"):
    """layers_stack for the port: list of (one_minus_n2 complex, z) in reference order."""
    L = lib("port")
    om = np.ascontiguousarray([[complex(l[0]).real, complex(l[0]).imag] for l in layers_stack],
                              dtype=np.float64)
    z = np.ascontiguousarray([l[1] for l in layers_stack], dtype=np.float64)
    tr = np.zeros(4)
    L.orc_parratt(C.c_int(len(z)), _p(om), _p(z), C.c_double(alpha), C.c_double(k0),
                  C.c_int(order), _p(tr))
    return complex(tr[0], tr[1]), complex(tr[2], tr[3])


def rot_axis(axis, angle):
    L = lib("port")
    r = np.zeros(9)
    L.orc_rot_axis(C.c_int(axis), C.c_double(angle), _p(r))
    return r.reshape(3, 3)


def rot_mul(a, b):
    L = lib("port")
    a = np.ascontiguousarray(a, dtype=np.float64).reshape(9)
    b = np.ascontiguousarray(b, dtype=np.float64).reshape(9)
    r = np.zeros(9)
    L.orc_rot_mul(_p(a), _p(b), _p(r))
    return r.reshape(3, 3)


def dwba_combine(fc, sf, ff, weight=1.0, intensity=None):
    L = lib("port")
    n = len(fc) // 4
    out = np.zeros(n) if intensity is None else np.ascontiguousarray(intensity, dtype=np.float64)
    fc, fcf = _cbuf(fc)
    sf, sff = _cbuf(sf)
    ff, fff = _cbuf(ff)
    L.orc_dwba_combine(C.c_int(n), _p(fcf), _p(sff), _p(fff), C.c_double(weight), _p(out))
    return out


def chi2(model, counts, mask=None, scale=1.0):
    L = lib("port")
    L.orc_chi2.restype = C.c_double
    m = np.ascontiguousarray(model, dtype=np.float64)
    c = np.ascontiguousarray(counts, dtype=np.float64)
    mk = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint32)
    return L.orc_chi2(C.c_int(len(m)), _p(m), _p(c),
                      None if mk is None else mk.ctypes.data_as(_up), C.c_double(scale))


def abs_diff_square(ref, data, mask):
    L = lib("port")
    L.orc_abs_diff_square.restype = C.c_double
    r = np.ascontiguousarray(ref, dtype=np.float64)
    d = np.ascontiguousarray(data, dtype=np.float64)
    mk = np.ascontiguousarray(mask, dtype=np.uint32)
    return L.orc_abs_diff_square(C.c_int(len(r)), _p(r), _p(d), mk.ctypes.data_as(_up))


def cylinder_params(radius, height, spread=0.0, nvalues=1):
    """Cylinder parameters; with spread > 0 a Gaussian over +-3 sigma sampled at nvalues points
    (param_distribution semantics; the reference sums these radii/heights unweighted)."""
    if spread > 0:
        sr, sh = spread * radius, spread * height
        return [dict(type="radius", stat="gaussian", min=radius - 3 * sr, max=radius + 3 * sr,
                     mean=radius, deviation=sr, nvalues=nvalues),
                dict(type="height", stat="gaussian", min=height - 3 * sh, max=height + 3 * sh,
                     mean=height, deviation=sh, nvalues=nvalues)]
    return [dict(type="radius", min=radius, max=radius, nvalues=1),
            dict(type="height", min=height, max=height, nvalues=1)]


def rel_err(a, b):
    """Norm-wise relative error ||a-b||_2 / ||b||_2 (the project's single error definition)."""
    a = np.asarray(a)
    b = np.asarray(b)
    den = float(np.linalg.norm(b.ravel()))
    return float(np.linalg.norm((a - b).ravel())) / (den if den > 0 else 1.0)


def smear_gaussian(image, sigma, backend="port"):
    """Convolutions::convolution_gaussian_2d of a (nrow, ncol) image (a copy is returned)."""
    L = lib(backend)
    img = np.ascontiguousarray(image, dtype=np.float64).copy()
    ny, nx = img.shape
    f = L.orc_smear_gaussian if backend == "port" else L.ref_smear_gaussian
    rc = f(_p(img), C.c_int(nx), C.c_int(ny), C.c_double(sigma))
    if rc != 0:
        raise RuntimeError("smear_gaussian failed")
    return img


def normalize(data):
    """HipGISAXS::normalize (a copy; the first element is left as it is)."""
    L = lib("port")
    d = np.ascontiguousarray(data, dtype=np.float64).copy()
    ok = L.orc_normalize(_p(d), C.c_long(d.size))
    return d, bool(ok)


def structure_sum(intensities, iratios):
    L = lib("port")
    I = np.ascontiguousarray(intensities, dtype=np.float64).reshape(len(iratios), -1)
    r = np.ascontiguousarray(iratios, dtype=np.float64)
    out = np.zeros(I.shape[1])
    L.orc_structure_sum(C.c_int(len(r)), C.c_long(I.shape[1]), _p(I), _p(r), _p(out))
    return out


def _libc_rand():
    libc = C.CDLL(None)
    libc.rand.restype = C.c_int
    return libc.rand


RAND_MAX = 2147483647  # glibc


def _read_obj_shape_def(path):
    """A Wavefront OBJ's vertices and triangles (v / f lines; f items v, v/vt, v/vt/vn, v//vn)
    turned into shape_def rows (mesh_to_shape_def)."""
    V, F = [], []
    with open(path) as f:
        for line in f:
            t = line.split()
            if not t:
                continue
            if t[0] == "v":
                V.append([float(x) for x in t[1:4]])
            elif t[0] == "f" and len(t) == 4:
                F.append([int(x.split("/")[0]) - 1 for x in t[1:4]])
    return mesh_to_shape_def(np.array(V), np.array(F, dtype=np.int32))


def _weight_gaussian(x, mean, sigma):
    """HipGISAXS::gaussian (include/sim/hipgisaxs_main.hpp:151-156)."""
    tiny, sqrt_2pi = 2.2250738585072014e-308, 2.506628
    if sigma < tiny:
        return 1.0 if x - mean < tiny else 0.0
    return 1.0 / (sigma * sqrt_2pi) * math.exp(-(x - mean) * (x - mean) / (2 * sigma * sigma))


def _weight_cauchy(x, l, sc):
    """HipGISAXS::cauchy (include/sim/hipgisaxs_main.hpp:169-172)."""
    tiny = 2.2250738585072014e-308
    if sc > tiny:
        return 1.0 / (3.141592653589793 * sc * (1.0 + ((x - l) / sc) * ((x - l) / sc)))
    return 0.0 if x - l > tiny else 1.0


def scale_plan(s, ngr, gw=None):
    """run_gisaxs's scaling and repetition loops (src/sim/hipgisaxs_main.cpp:815-870,
    1017-1040) with construct_scaling_distribution (:2179-2226), construct_repetition_
    distribution (:2100-2176) and generate_repetition_range (:2089-2098): per grain the list
    of (a, b, c scaled, repetitions, weight) in the reference's order."""
    stat, mean, sd0, ns = s["scaling_stat"], s["scaling_mean"], s["scaling_stddev"], s["scaling_nsamples"]
    nv = [1 if (stat[i] == "none" or sd0[i] == 0) else int(ns[i]) for i in range(3)]
    dist_branch = any(sd0[i] > 0 for i in range(3))  # grain_scaling_is_dist()
    rnd = woo_mt_rand()
    width, max_nvals = 4, max(nv)
    samples, weights = [], []
    for i in range(3):
        sd = sd0[i] if stat[i] != "none" else 0.0
        if stat[i] == "none":
            samples.append(mean[i]); weights.append(1.0)
        elif stat[i] in ("gaussian", "cauchy"):
            mn = mean[i] - width * sd
            dx = (2 * width) * sd / (max_nvals + 1)
            for j in range(max_nvals):
                t = mn + j * dx + rnd() * dx
                samples.append(t)
                weights.append(_weight_gaussian(t, mean[i], sd) if stat[i] == "gaussian"
                               else _weight_cauchy(t, mean[i], sd))
        else:
            raise ValueError(stat[i])
    if s["repetition_dist"]:
        nrep = len(samples) if len(samples) > 1 else ngr
        vals = []
        for ax in ("xrepetition", "yrepetition", "zrepetition"):
            r = s[ax]
            if r["stat"] == "none":
                vals.append([r["min"]])
            else:
                rr = woo_mt_rand()  # a fresh generator per axis
                vals.append([int(r["min"] + rr() * float(r["max"] - r["min"])) for _ in range(nrep)])
        sizes = min(len(v) for v in vals)
        repeats = [(float(vals[0][i]), float(vals[1][i]), float(vals[2][i])) for i in range(sizes)]
    else:
        repeats = [tuple(s["repetition"])]
    num_scaling, num_repeats = len(samples) // 3, len(repeats)
    if num_scaling == num_repeats:
        nscale = num_scaling
    elif num_scaling == 1:
        nscale = num_repeats
    elif num_repeats == 1:
        nscale = num_scaling
    else:
        raise ValueError("scaling and repetition counts differ")
    lat = s["lattice"]
    plan = []
    for g in range(ngr):
        row = []
        for i in range(nscale):
            if dist_branch:
                sc = [samples[i + num_scaling * k] for k in range(3)]
                w = weights[i]
            else:
                sc = samples[:3]
                w = weights[0]
            rp = repeats[g % num_repeats if s["repetition_dist"] else 0]
            abc = np.array([[v * sc[0] for v in lat["a"]], [v * sc[1] for v in lat["b"]],
                            [v * sc[2] for v in lat["c"]]])
            row.append((abc, [1.0 if x < 1 else x for x in rp], (1.0 if gw is None else gw[g]) * w))
        plan.append(row)
    return plan


def compute_gisaxs(hig, hig_dir=".", rand=None, alpha_i=None, phi=None):
    """HipGISAXS::compute_gisaxs / run_gisaxs (src/sim/hipgisaxs_main.cpp:630-1440) for the
    configurations hgx_hig_compute_gisaxs supports, composed from this oracle's pinned pieces
    (QGrid, MultiLayer::propagation_coeffs, the analytic and numeric form factors, the
    structure factors, the DWBA combination and the structure sum).  `hig`: the reader's
    JSON model (dict).  Orientations drawn by "range"/"random" call `rand` (default: the C
    library's rand()) in the reference's order.  alpha_i, phi: a scan point's angles in
    degrees (run_all_gisaxs, :283-613; default: the first of each): the detector grid stays
    the first alpha_i's (HipGISAXS::init), qz_extended and the Fresnel coefficients take this
    alpha_i (layer_qgrid_qz, propagation_coeffs, :779-785), the structures this phi.  Returns
    the nrow x ncol image (FP64)."""
    rand = rand or _libc_rand()
    sc, cp = hig["scattering"], hig["computation"]
    saxs = sc["expt"] == "saxs"
    value, unit = sc["photon_value"], sc["photon_unit"]
    kev = value / 1000 if unit == "ev" else value  # HipGISAXS::init, :146-160
    ncol, nrow = int(cp["resolution"][0]), int(cp["resolution"][1])
    (ymin, zmin), (ymax, zmax) = cp["minpoint"], cp["maxpoint"]
    G = Grid(ncol, nrow, ymin, zmin, ymax, zmax, sc["alphai"][0], kev, (0.0, 0.0))
    if alpha_i is not None and alpha_i * 3.141592653589793 / 180 != G.alpha_i:
        G.reextend(alpha_i)
    layers = [(l["refindex"][0], l["refindex"][1], l["thickness"], l["order"])
              for _, l in sorted(hig["layers"].items(), key=lambda kv: int(kv[0]))]
    fc = propagation_coeffs(G, layers, 0)  # particle layer order 0 (:779-785)
    pi = 3.141592653589793
    rot_phi = rot_axis(2, (sc["inplanerot"][0] if phi is None else phi) * pi / 180)
    meshes = {}
    for key, sh in hig["shapes"].items():
        if sh["name"] == "custom":
            p = sh["name_str"]
            if not os.path.exists(p) and not os.path.isabs(p):
                p = os.path.join(hig_dir, p)
            meshes[key] = _read_obj_shape_def(p)
    intens = []
    for skey, s in hig["structures"].items():  # key order, as the product walks them
        uc = hig["unitcells"][s["unitcell_key"]]
        # spatial_distribution "regular" (:1765-1828), cell_ = 0, tz = 0
        nd = [float(v) for v in s["maxgrains"]]
        n0, n1, n2 = int(nd[0]), int(nd[1]), int(nd[2])
        ngr = int(nd[0] * nd[1] * nd[2])
        sp = s["spacing"]
        axes = []
        for k in range(3):
            n_k, st = (n0, n1, n2)[k], sp[k]
            mx = st * (nd[k] - 1)
            vals, val = [], 0.0
            for _ in range(n_k):
                vals.append(val - mx / 2 if k < 2 else val + 0.0)
                val += st
            axes.append(vals)
        d = np.zeros((3, ngr))
        for x in range(n0):
            for y in range(n1):
                for z in range(n2):
                    g = n1 * n2 * x + n2 * y + z
                    d[0, g], d[1, g], d[2, g] = axes[0][x], axes[1][y], axes[2][z]
        # orientation_distribution (:1869-1960)
        rots = []
        for name in ("rot1", "rot2", "rot3"):
            r = s[name]
            rots.append((0.0, 0.0, 0.0) if r["axis"] == "n" else
                        (float(ord(r["axis"]) - ord("x")), r["angles"][0], r["angles"][1]))
        nn = np.zeros((3, ngr))
        wg = np.ones((3, ngr))
        stat = s["orientation_stat"]
        if stat == "single":
            for k in range(3):
                nn[k, :] = rots[k][1] * pi / 180
        elif stat == "random":
            for x in range(3 * ngr):
                nn.reshape(-1)[x] = (float(rand()) / RAND_MAX) * 2 * pi
        elif stat == "range":
            for k in range(3):
                dr = abs(rots[k][2] - rots[k][1])
                for x in range(ngr):
                    nn[k, x] = (rots[k][1] + (float(rand()) / RAND_MAX) * dr) * pi / 180
        elif stat in ("gaussian", "normal", "cauchy"):
            # evenly stepped angles, weighted by the distribution (:1920-2082)
            tiny = 2.2250738585072014e-308
            robj = (s["rot1"], s["rot2"], s["rot3"])
            for k in range(3):
                span = abs(rots[k][2] - rots[k][1])
                dr = span / ngr if stat != "cauchy" else (span / (ngr - 1) if ngr > 1 else float("nan"))
                if dr > tiny:
                    for x in range(ngr):
                        t = rots[k][1] + x * dr
                        nn[k, x] = t * pi / 180
                        wg[k, x] = (_weight_cauchy(t, robj[k]["location"], robj[k]["scale"]) if stat == "cauchy"
                                    else _weight_gaussian(t, robj[k]["mean"], robj[k]["sd"]))
                else:
                    nn[k, :] = rots[k][1] * pi / 180
        else:
            raise ValueError(stat)
        gw = [wg[0, g] * wg[1, g] * wg[2, g] if stat in ("gaussian", "cauchy") else 1.0
              for g in range(ngr)]
        lat = s["lattice"]
        plan = scale_plan(s, ngr, gw)
        I = np.zeros(G.n)
        for gi in range(ngr):
            rot = rot_mul(rot_mul(rot_mul(rot_phi, rot_axis(int(rots[2][0]), nn[2, gi])),
                                  rot_axis(int(rots[1][0]), nn[1, gi])),
                          rot_axis(int(rots[0][0]), nn[0, gi]))
            dv = d[:, gi]
            center = np.array([rot[i, 0] * dv[0] + rot[i, 1] * dv[1] + rot[i, 2] * dv[2]
                               for i in range(3)]) + np.array(s["transvec"])
            ff = np.zeros(4 * G.n, dtype=np.complex128)
            for ekey in uc:
                sh = hig["shapes"][ekey]
                zr, yr, xr = sh["rot"]
                srot = rot_mul(rot_mul(rot_mul(rot, rot_axis(0, xr)), rot_axis(1, yr)), rot_axis(2, zr))
                dn2 = complex(0.0 - 2 * sh["refindex"][0], 0.0 - 2 * sh["refindex"][1])
                params = [{"type": p["type"], "stat": p["stat"], "min": p["min"], "max": p["max"],
                           "mean": p["p1"], "deviation": p["p2"], "nvalues": p["nvalues"]}
                          for p in sh["params"].values()]
                for loc in uc[ekey]:
                    if sh["name"] == "custom":
                        eff = ff_approx_triangle(meshes[ekey], G.qx, G.qy, G.qz_ext, srot)
                    else:
                        eff = ff_analytic(G, sh["name"], params, transvec=loc, rot=srot)
                    ff = ff + dn2 * eff
            for abc, rp, w in plan[gi]:
                if s["type"] == "paracrystal":
                    pc = s["paracrystal"]
                    sf = sf_paracrystal(G, pc["dims"], LATTICE.get(lat["type"], 1), pc.get("xmean", 0.0),
                                        pc.get("ymean", 0.0), pc.get("xstddev", 0.0),
                                        pc.get("ystddev", 0.0), pc.get("domain", 0.0))
                elif s["type"] == "percusyevick":
                    py = s["percusyevick"]
                    sf = sf_percus_yevick(G, py["diameter"], py["volfraction"], py["dims"])
                elif saxs:  # the detector's real qz (sf.cpp:199-200)
                    sf = sf_lattice_arrays(abc, rp, (1.0, 1.0, 1.0), center, rot, G.qx, G.qy,
                                           G.qz.astype(np.complex128))
                else:
                    sf = sf_lattice(G, abc, rp, (1.0, 1.0, 1.0), center, rot)
                if saxs:  # run_gisaxs :1099-1103: assigned, not added; the first N values
                    t = (w * sf[:G.n]) * ff[:G.n]
                    I = t.real * t.real + t.imag * t.imag
                else:
                    I = dwba_combine(fc, sf, ff, w, I)
        intens.append(I)
    ratios = [s["iratio"] for s in hig["structures"].values()]
    img = structure_sum(np.array(intens), ratios)
    return img.reshape(nrow, ncol)


class MT19937_64:
    """The 64-bit Mersenne Twister of Matsumoto and Nishimura (std::mt19937_64: n = 312,
    m = 156, r = 31 and the standard's tempering constants), restated from the published
    algorithm."""

    N, M = 312, 156
    MATRIX_A = 0xB5026F5AA96619E9
    UM, LM = 0xFFFFFFFF80000000, 0x7FFFFFFF
    MASK = (1 << 64) - 1

    def __init__(self, seed=0):
        self.mt = [0] * self.N
        self.mt[0] = seed & self.MASK
        for i in range(1, self.N):
            x = self.mt[i - 1]
            self.mt[i] = (6364136223846793005 * (x ^ (x >> 62)) + i) & self.MASK
        self.i = self.N

    def __call__(self):
        if self.i >= self.N:
            mt = self.mt
            for k in range(self.N):
                x = (mt[k] & self.UM) | (mt[(k + 1) % self.N] & self.LM)
                y = x >> 1
                if x & 1:
                    y ^= self.MATRIX_A
                mt[k] = mt[(k + self.M) % self.N] ^ y
            self.i = 0
        y = self.mt[self.i]
        self.i += 1
        y ^= (y >> 29) & 0x5555555555555555
        y ^= (y << 17) & 0x71D67FFFEDA60000
        y ^= (y << 37) & 0xFFF7EEE000000000
        y ^= y >> 43
        return y & self.MASK


def woo_mt_rand():
    """woo::MTRandomNumberGenerator (include/woo/random/woo_mtrandom.hpp): seed 0, rand() =
    (x - min) / (max - min) in doubles."""
    g = MT19937_64(0)
    mx = float((1 << 64) - 1)
    return lambda: (float(g()) - 0.0) / (mx - 0.0)


FIT_METRICS = {"sqrt_unit_l2": 0, "sqrt_c_l2": 1, "cbrt_unit_l2": 2, "cbrt_c_l2": 3,
               "sqrt_unit_l2_residual": 4, "sqrt_c_l2_residual": 5, "sqrt_unit_l1": 6,
               "cbrt_unit_l1": 7}


def fit_distance(metric, ref, data, mask=None, backend="port"):
    """The fitter's distance measure `metric` (name or number): an array of 1 value, or n for
    the residual forms."""
    m = FIT_METRICS.get(metric, metric)
    L = lib(backend)
    r = np.ascontiguousarray(ref, dtype=np.float64).ravel()
    d = np.ascontiguousarray(data, dtype=np.float64).ravel()
    mk = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint32).ravel()
    out = np.zeros(r.size)
    f = L.orc_fit_distance if backend == "port" else L.ref_fit_distance
    f.restype = C.c_long
    k = f(C.c_int(int(m)), C.c_long(r.size), _p(r), _p(d),
          None if mk is None else mk.ctypes.data_as(_up), _p(out))
    if k < 0:
        raise ValueError(f"fit_distance({metric}) failed")
    return out[:k].copy()
