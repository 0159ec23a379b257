"""HiG input files: HiGInput (include/config/hig_input.hpp) over the C reader (hgx_hig_read).

    inp = read_hig("cylinders.hig")
    inp.shapes["s1"]["params"]["radius"]["min"]
    k0, alpha_i, freq = inp.beam()
    grid = inp.qgrid(ctx)          # QGrid::create + create_qz_extended on the device

The description is the reader's JSON (hgx_hig_json) as plain dicts; the accessor methods
carry the reference's names (scattering_alphai, param_resolution, ...).  Parsing is host
work and needs no GPU; qgrid() builds device arrays.
"""
from __future__ import annotations

import ctypes as C
import json
import os

import numpy as np

from ._capi import check, lib
from .core import PRECISION, Context, QGrid, _in, _is_tensor

# the fitting block's distance metrics (hgx_fit_metric)
METRICS = {"sqrt_unit_l2": 0, "sqrt_c_l2": 1, "cbrt_unit_l2": 2, "cbrt_c_l2": 3,
           "sqrt_unit_l2_residual": 4, "sqrt_c_l2_residual": 5, "sqrt_unit_l1": 6,
           "cbrt_unit_l1": 7}


class HiGInput:
    """A HiG file read by hgx_hig_read (HiGInput::construct_input_config)."""

    def __init__(self, path: str):
        h = C.c_void_p()
        check(lib().hgx_hig_read(os.fsencode(path), C.byref(h)))
        self._h = h
        self.path = path
        self._reload()

    def _reload(self):
        n = C.c_size_t()
        check(lib().hgx_hig_json(self._h, None, 0, C.byref(n)))
        buf = C.create_string_buffer(n.value + 1)
        check(lib().hgx_hig_json(self._h, buf, n.value + 1, C.byref(n)))
        self.data = json.loads(buf.value.decode())

    # the blocks of the file
    @property
    def shapes(self):
        return self.data["shapes"]

    @property
    def layers(self):
        """{order: layer}, sorted by order as the reference's std::map keeps them."""
        return {int(k): v for k, v in sorted(self.data["layers"].items(), key=lambda kv: int(kv[0]))}

    @property
    def unitcells(self):
        return self.data["unitcells"]

    @property
    def structures(self):
        return self.data["structures"]

    @property
    def scattering(self):
        return self.data["scattering"]

    @property
    def detector(self):
        return self.data["detector"]

    @property
    def compute(self):
        return self.data["computation"]

    @property
    def fit_params(self):
        return self.data["fitparams"]

    @property
    def algorithms(self):
        return self.data["algorithms"]

    # accessors with the reference's names (include/config/hig_input.hpp:170-260)
    def scattering_alphai(self):
        return tuple(self.scattering["alphai"])

    def scattering_inplanerot(self):
        return tuple(self.scattering["inplanerot"])

    def scattering_tilt(self):
        return tuple(self.scattering["tilt"])

    def photon_energy(self):
        return self.scattering["photon_value"], self.scattering["photon_unit"]

    def param_resolution(self):
        return [int(v) for v in self.compute["resolution"]]

    def param_output_minpoint(self):
        return tuple(self.compute["minpoint"])

    def param_output_maxpoint(self):
        return tuple(self.compute["maxpoint"])

    def param_output_type(self):
        return self.compute["region_type"]

    def num_structures(self):
        return len(self.structures)

    def substrate_refindex(self):
        sub = self.layers.get(-1)
        return (sub["refindex"][0], sub["refindex"][1]) if sub else (0.0, 0.0)

    def fit_param_keys(self):
        return sorted(self.fit_params)

    # device set-up of HipGISAXS::init
    def beam(self):
        """(k0 in 1/nm, alpha_i in radians, frequency) as HipGISAXS::init computes them."""
        k0, ai, fr = C.c_double(), C.c_double(), C.c_double()
        check(lib().hgx_hig_beam(self._h, C.byref(k0), C.byref(ai), C.byref(fr)))
        return k0.value, ai.value, fr.value

    def qgrid(self, ctx: Context, dn2=(0.0, 0.0)) -> QGrid:
        """The computation block's q-space grid with its DWBA extension for dn2 (device)."""
        h = C.c_void_p()
        check(lib().hgx_hig_qgrid(ctx.handle, self._h, float(dn2[0]), float(dn2[1]), C.byref(h)))
        return QGrid(ctx, h)

    def image_size(self):
        """(nrow, ncol) of the detector image (computation.resolution)."""
        r, c = C.c_int(), C.c_int()
        check(lib().hgx_hig_image_size(self._h, C.byref(r), C.byref(c)))
        return r.value, c.value

    def compute_gisaxs(self, ctx: Context, precision: str = "f64", out=None):
        """HipGISAXS::compute_gisaxs on the device (hgx_hig_compute_gisaxs): the nrow x ncol
        intensity image of every structure's grains, summed with the iratios.  `out`: a
        float64 numpy array or CUDA tensor of nrow*ncol values (allocated when None).
        precision "f32c" computes mesh form factors in compensated FP32, and on grids with
        real qz the fused grain kernel's cylinder, sphere and box cells and lattice structure
        factors in FP32C (FP64 phases, FP32 transcendentals and sums).  expt "saxs" takes the
        reference's Born branch (each structure keeps its last grain's last scaling sample, as
        the reference's assignment leaves it); nslices > 1 gives the reference's zero image;
        a description with angle scans is refused (compute_scan_point runs them)."""
        nrow, ncol = self.image_size()
        if out is None:
            out = np.zeros((nrow, ncol))
        ptr = out.data_ptr() if _is_tensor(out) else out.ctypes.data
        check(lib().hgx_hig_compute_gisaxs(ctx.handle, self._h, PRECISION[precision], C.c_void_p(ptr)))
        return out

    # angle scans (HipGISAXS::run_all_gisaxs)
    def scan_size(self):
        """(n_alphai, n_phi, n_tilt) of the scattering block's scans."""
        a, p, t = C.c_int(), C.c_int(), C.c_int()
        check(lib().hgx_hig_scan_size(self._h, C.byref(a), C.byref(p), C.byref(t)))
        return a.value, p.value, t.value

    def scan_points(self):
        """[(alpha_i, phi, tilt)] in degrees, in the reference's loop order."""
        na, nph, nt = self.scan_size()
        out = []
        for i in range(na * nph * nt):
            a, p, t = C.c_double(), C.c_double(), C.c_double()
            check(lib().hgx_hig_scan_point(self._h, i, C.byref(a), C.byref(p), C.byref(t)))
            out.append((a.value, p.value, t.value))
        return out

    def compute_scan_point(self, ctx: Context, p: int, precision: str = "f64", out=None):
        """The image of scan point p (hgx_hig_compute_scan_point)."""
        nrow, ncol = self.image_size()
        if out is None:
            out = np.zeros((nrow, ncol))
        ptr = out.data_ptr() if _is_tensor(out) else out.ctypes.data
        check(lib().hgx_hig_compute_scan_point(ctx.handle, self._h, PRECISION[precision], int(p),
                                               C.c_void_p(ptr)))
        return out

    def run_all_gisaxs(self, ctx: Context, precision: str = "f64"):
        """Every scan point's image and, per alpha_i with more than one phi or tilt, their sum
        (the reference's "averaged" output): (images [(alpha_i, phi, tilt, image)],
        sums {alpha_i: image})."""
        na, nph, nt = self.scan_size()
        images, sums = [], {}
        for i, (a, p, t) in enumerate(self.scan_points()):
            img = self.compute_scan_point(ctx, i, precision)
            images.append((a, p, t, img))
            if nph > 1 or nt > 1:
                sums[a] = img.copy() if a not in sums else sums[a] + img
        return images, sums

    # fitting (HiGInput::update_params, HipGISAXSObjectiveFunction)
    def fit_keys(self):
        """The fit parameters' keys in the order of an x vector (fit_param_keys)."""
        n = C.c_int()
        check(lib().hgx_hig_fit_count(self._h, C.byref(n)))
        keys = []
        for i in range(n.value):
            k = C.create_string_buffer(256)
            check(lib().hgx_hig_fit_param(self._h, i, k, 256, None, 0, None, None))
            keys.append(k.value.decode())
        return keys

    def fit_reference(self):
        """The referencedata block: {"path", "mask", "npar", "nperp"} (reference_data_path,
        reference_data_mask; paths as written, "" when not given)."""
        p, m = C.create_string_buffer(4096), C.create_string_buffer(4096)
        npar, nperp = C.c_int(), C.c_int()
        check(lib().hgx_hig_fit_reference(self._h, 0, p, 4096, m, 4096, C.byref(npar), C.byref(nperp)))
        return {"path": p.value.decode(), "mask": m.value.decode(), "npar": npar.value,
                "nperp": nperp.value}

    def override_qregion(self, ny: int, nz: int, i: int = 0):
        """HipGISAXS::override_qregion: the simulation re-gridded to an ny x nz reference image
        over the referencedata block's fit region."""
        check(lib().hgx_hig_override_qregion(self._h, int(ny), int(nz), int(i)))
        self._reload()

    def fit_algorithms(self):
        """The analysis algorithms in file order: [{"name", "metric", "tolerance",
        "regularization"}], metric an hgx_fit_metric number (-1: none of them)."""
        n = C.c_int()
        check(lib().hgx_hig_fit_algorithm_count(self._h, C.byref(n)))
        out = []
        for i in range(n.value):
            nm = C.create_string_buffer(64)
            met, tol, reg = C.c_int(), C.c_double(), C.c_double()
            check(lib().hgx_hig_fit_algorithm(self._h, i, nm, 64, C.byref(met), C.byref(tol), C.byref(reg)))
            out.append({"name": nm.value.decode(), "metric": met.value, "tolerance": tol.value,
                        "regularization": reg.value})
        return out

    def update_param(self, variable: str, value: float):
        """Sets one parameter by its variable name, e.g. "shape['s1']:param['radius']:min"."""
        check(lib().hgx_hig_update_param(self._h, variable.encode(), float(value)))
        self._reload()

    def fit_update(self, x):
        """Sets every fit parameter: x[i] for fit_keys()[i]."""
        xa = np.ascontiguousarray(x, dtype=np.float64).ravel()
        check(lib().hgx_hig_fit_update(self._h, xa.ctypes.data, int(xa.size)))
        self._reload()

    def objective(self, ctx: Context, x, ref, mask=None, metric="sqrt_unit_l2", reg_alpha=0.0):
        """HipGISAXSObjectiveFunction::operator()(x) on the device: the distance between the
        simulation at x and `ref` (nrow x ncol), regularised; a numpy array of 1 value, or one
        per pixel for the residual metrics."""
        xa = np.ascontiguousarray(x, dtype=np.float64).ravel()
        pr, kr = _in(ref, np.float64)
        pm, km = (None, None) if mask is None else _in(mask, np.uint32)
        nrow, ncol = self.image_size()
        dist = np.zeros(nrow * ncol)
        nd = C.c_long()
        check(lib().hgx_hig_objective(ctx.handle, self._h, xa.ctypes.data, int(xa.size), pr, pm,
                                      METRICS.get(metric, metric), float(reg_alpha),
                                      dist.ctypes.data, C.byref(nd)))
        self._reload()
        return dist[:nd.value].copy()

    def objective_grad(self, ctx: Context, x, ref, mask=None, metric="sqrt_unit_l2", reg_alpha=0.0):
        """(distance, gradient) of the objective at x for a scalar distance measure: the
        gradient by the tangent of the simulation (hgx_hig_objective_grad), one value per fit
        parameter in fit_keys() order."""
        xa = np.ascontiguousarray(x, dtype=np.float64).ravel()
        pr, kr = _in(ref, np.float64)
        pm, km = (None, None) if mask is None else _in(mask, np.uint32)
        dist = np.zeros(1)
        grad = np.zeros(xa.size)
        check(lib().hgx_hig_objective_grad(ctx.handle, self._h, xa.ctypes.data, int(xa.size), pr, pm,
                                           METRICS.get(metric, metric), float(reg_alpha),
                                           dist.ctypes.data, grad.ctypes.data))
        self._reload()
        return float(dist[0]), grad

    def population(self, ctx: Context, npop: int, ref, mask=None, metric="sqrt_unit_l2", reg_alpha=0.0,
                   precision: str = "f64"):
        """A fitting population of this description (hgx_hig_population_*): evaluates npop
        parameter vectors per call, each distance the one objective() returns for it."""
        return HiGPopulation(ctx, self, npop, ref, mask, metric, reg_alpha, precision)

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None):
            lib().hgx_hig_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def read_hig(path: str) -> HiGInput:
    return HiGInput(path)


def fit_distance(ctx: Context, metric, ref, data, mask=None):
    """hgx_fit_distance: the fitter's distance measure (name or number) between two images."""
    m = METRICS.get(metric, metric)
    pr, kr = _in(ref, np.float64)
    pd, kd = _in(data, np.float64)
    n = int(kr.numel() if _is_tensor(kr) else kr.size)
    pm, km = (None, None) if mask is None else _in(mask, np.uint32)
    out = np.zeros(n if m in (4, 5) else 1)
    check(lib().hgx_fit_distance(ctx.handle, int(m), n, pr, pd, pm, out.ctypes.data))
    return out


def read_image(path: str):
    """hgx_read_image: a reference image (text or EDF) as (values, ncol, nrow); values may hold
    a last row more than ncol x nrow counts, as the reference's text reader leaves it."""
    cnt, nc, nr = C.c_long(), C.c_int(), C.c_int()
    check(lib().hgx_read_image(os.fsencode(path), None, 0, C.byref(cnt), C.byref(nc), C.byref(nr)))
    data = np.zeros(cnt.value)
    check(lib().hgx_read_image(os.fsencode(path), data.ctypes.data, cnt.value, C.byref(cnt),
                               C.byref(nc), C.byref(nr)))
    return data, nc.value, nr.value


def read_mask(path: str):
    """hgx_read_mask: a fit mask (text or EDF) as uint32 values."""
    cnt = C.c_long()
    check(lib().hgx_read_mask(os.fsencode(path), None, 0, C.byref(cnt)))
    m = np.zeros(cnt.value, dtype=np.uint32)
    check(lib().hgx_read_mask(os.fsencode(path), m.ctypes.data, cnt.value, C.byref(cnt)))
    return m


class HiGPopulation:
    """hgx_hig_population: the particle loop of the reference's PSO fitter
    (src/analyzer/hipgisaxs_fit_pso.cpp:521-545) for npop candidates per evaluation, on a copy
    of the description taken at creation."""

    def __init__(self, ctx: Context, d: HiGInput, npop: int, ref, mask=None, metric="sqrt_unit_l2",
                 reg_alpha=0.0, precision: str = "f64"):
        pr, kr = _in(ref, np.float64)
        pm, km = (None, None) if mask is None else _in(mask, np.uint32)
        h = C.c_void_p()
        check(lib().hgx_hig_population_create(ctx.handle, d.handle, int(npop), pr, pm,
                                              METRICS.get(metric, metric), float(reg_alpha),
                                              PRECISION[precision], C.byref(h)))
        self._h = h
        self.npop = int(npop)
        self.nx = len(d.fit_keys())

    def eval(self, X) -> np.ndarray:
        """Distances of the npop rows of X (npop x nx, fit_keys() order per row)."""
        Xa = np.ascontiguousarray(X, dtype=np.float64).reshape(self.npop, self.nx)
        dist = np.zeros(self.npop)
        check(lib().hgx_hig_population_eval(self._h, Xa.ctypes.data, int(self.nx), dist.ctypes.data))
        return dist

    def close(self):
        if getattr(self, "_h", None):
            lib().hgx_hig_population_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
