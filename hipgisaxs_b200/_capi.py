"""ctypes bindings to libhgx.so (the C ABI declared in include/hgx.h).

The library is built in-tree (python -m hipgisaxs_b200.build).  Loading fails loudly when
it is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhgx.so")

HGX_OK = 0
F64, F32C = 0, 1
C128, C64 = 0, 1

_vp = C.c_void_p
_i = C.c_int
_d = C.c_double

# name -> (restype, argtypes)
SIGNATURES = {
    "hgx_last_error": (C.c_char_p, []),
    "hgx_status_string": (C.c_char_p, [_i]),
    "hgx_version": (_i, []),
    "hgx_create": (_i, [_i, C.POINTER(_vp)]),
    "hgx_destroy": (_i, [_vp]),
    "hgx_set_stream": (_i, [_vp, _vp]),
    "hgx_get_stream": (_vp, [_vp]),
    "hgx_synchronize": (_i, [_vp]),
    "hgx_qgrid_from_arrays": (_i, [_vp, _i, _vp, _vp, _i, _vp, _i, C.POINTER(_vp)]),
    "hgx_qgrid_create": (_i, [_vp, _i, _i, _d, _d, _d, _d, _d, _d, _d, _d, C.POINTER(_vp)]),
    "hgx_qgrid_read": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "hgx_qgrid_info": (_i, [_vp, C.POINTER(_i), C.POINTER(_i), C.POINTER(_i), C.POINTER(_i),
                            C.POINTER(_i)]),
    "hgx_qgrid_destroy": (_i, [_vp]),
    "hgx_ff_triangles_q": (_i, [_vp, _vp, _vp, _i, _vp, _i, _vp, _i]),
    "hgx_ff_triangles_q_ex": (_i, [_vp, _vp, _vp, _i, _vp, _i, _vp, _i, _i]),
    "hgx_ff_tune": (_i, [_vp, _vp, _vp, _i, _vp, _i, _i, C.POINTER(_i), C.POINTER(_d), _vp]),
    "hgx_ff_triangles": (_i, [_vp, _vp, _i, _i, _vp, _vp, _i, _vp, _vp, _i, _vp]),
    "hgx_ff_exact_triangles_q": (_i, [_vp, _vp, _vp, _i, _vp, _vp, _i]),
    "hgx_ff_exact_triangles": (_i, [_vp, _vp, _i, _i, _vp, _vp, _i, _vp, _vp, _vp]),
    "hgx_param_distribution": (_i, [_i, _d, _d, _d, _d, _i, _vp, _vp, _i, C.POINTER(_i)]),
    "hgx_ff_analytic": (_i, [_vp, _vp, _i, _i, _vp, _vp, _i, _vp, _vp, _i, _vp, _vp, _i, _vp,
                             _vp, _d, _d, _vp, _vp, _vp, _i]),
    "hgx_ff_analytic_ex": (_i, [_vp, _vp, _i, _i, _vp, _vp, _i, _vp, _vp, _i, _vp, _vp, _i, _vp,
                             _vp, _d, _d, _vp, _vp, _vp, _i, _i]),
    "hgx_ff_analytic_params": (_i, [_vp, _vp, _i, _i, _vp, _d, _d, _vp, _vp, _vp, _i]),
    "hgx_ff_analytic_params_ex": (_i, [_vp, _vp, _i, _i, _vp, _d, _d, _vp, _vp, _vp, _i, _i]),
    "hgx_lattice_vectors": (_i, [_i, C.c_char_p, _vp, _vp]),
    "hgx_sf_lattice": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i]),
    "hgx_sf_lattice_ex": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i, _i]),
    "hgx_sf_paracrystal": (_i, [_vp, _vp, _i, _i, _d, _d, _d, _d, _d, _vp, _i]),
    "hgx_sf_percus_yevick": (_i, [_vp, _vp, _d, _d, _i, _vp, _i]),
    "hgx_propagation_coeffs": (_i, [_vp, _vp, _i, _vp, _vp, _vp, _vp, _d, _d, _i, _vp, _vp, _i]),
    "hgx_dwba_combine": (_i, [_vp, C.c_long, _vp, _vp, _vp, _i, _d, _vp]),
    "hgx_dwba_mesh_grains": (_i, [_vp, _vp, _vp, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _d, _d,
                                  _i, _vp]),
    "hgx_abs_diff_square": (_i, [_vp, C.c_long, _vp, _vp, _vp, _vp]),
    "hgx_residual_vector": (_i, [_vp, C.c_long, _vp, _vp, _vp, _vp]),
    "hgx_chi2": (_i, [_vp, C.c_long, _vp, _vp, _vp, _d, _vp]),
    "hgx_dwba_analytic_grains": (_i, [_vp, _vp, _i, _i, _vp, _d, _d, _vp, _i, _vp, _vp, _vp, _vp,
                                      _vp, _vp, _vp, _d, _d, _vp]),
    "hgx_structure_sum": (_i, [_vp, _i, C.c_long, _vp, _vp, _vp]),
    "hgx_gaussian_smearing": (_i, [_vp, _vp, _i, _i, _d]),
    "hgx_normalize": (_i, [_vp, _vp, C.c_long, C.POINTER(_i)]),
    "hgx_save_gisaxs": (_i, [_vp, _vp, _i, _i, C.c_char_p]),
    "hgx_cyl_batch_create": (_i, [_vp, _vp, _vp, _vp, _i, _vp, _vp, _vp, _d, _i, C.POINTER(_vp)]),
    "hgx_cyl_batch_eval": (_i, [_vp, _vp, _vp]),
    "hgx_cyl_batch_forward": (_i, [_vp, _vp, _vp]),
    "hgx_cyl_plain_forward": (_i, [_vp, _i, _vp, _vp]),
    "hgx_cyl_batch_info": (_i, [_vp, C.POINTER(C.c_long), C.POINTER(C.c_long)]),
    "hgx_cyl_batch_destroy": (_i, [_vp]),
    "hgx_cyl_shape_info": (_i, [_i, C.POINTER(_i), C.POINTER(_i)]),
    "hgx_cyl_batch_set_shape": (_i, [_vp, _i]),
    "hgx_cyl_batch_get_shape": (_i, [_vp, C.POINTER(_i)]),
    "hgx_cyl_batch_tune": (_i, [_vp, _vp, _i, C.POINTER(_i), C.POINTER(_d), _vp]),
    "hgx_obj_load": (_i, [C.c_char_p, C.POINTER(_vp)]),
    "hgx_mesh_info": (_i, [_vp, C.POINTER(_i), C.POINTER(_i), C.POINTER(_i), C.POINTER(_i)]),
    "hgx_mesh_read": (_i, [_vp, _vp, _vp]),
    "hgx_mesh_destroy": (_i, [_vp]),
    "hgx_read_shapes_file": (_i, [_vp, C.c_char_p, _vp, _i, C.POINTER(_i)]),
    "hgx_mesh_to_shape_def": (_i, [_vp, _i, _vp, _i, _vp, _vp]),
    "hgx_mesh_chi2_grad": (_i, [_vp, _vp, _i, _vp, _i, _vp, _vp, _vp, _d, _d, _d, _vp, _vp, _d,
                                _vp, _vp, _vp]),
    "hgx_mesh_chi2_grad_ex": (_i, [_vp, _vp, _i, _vp, _i, _vp, _vp, _vp, _d, _d, _d, _vp, _vp, _d,
                                _vp, _vp, _vp, _i]),
    "hgx_ff_triangles_noalloc": (_i, [_vp, _i, _i, _vp, _vp, _i, _vp, _vp, _vp, _i, _vp]),
    "hgx_ff_triangles_noalloc_status": (_i, [_vp, _vp]),
    "hgx_hig_read": (_i, [C.c_char_p, C.POINTER(_vp)]),
    "hgx_hig_json": (_i, [_vp, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    "hgx_hig_destroy": (_i, [_vp]),
    "hgx_hig_beam": (_i, [_vp, C.POINTER(_d), C.POINTER(_d), C.POINTER(_d)]),
    "hgx_hig_qgrid": (_i, [_vp, _vp, _d, _d, C.POINTER(_vp)]),
    "hgx_hig_image_size": (_i, [_vp, C.POINTER(_i), C.POINTER(_i)]),
    "hgx_hig_compute_gisaxs": (_i, [_vp, _vp, _i, _vp]),
    "hgx_hig_output_names": (_i, [_vp, C.c_char_p, C.c_size_t, C.c_char_p, C.c_size_t]),
    "hgx_hig_scan_size": (_i, [_vp, _vp, _vp, _vp]),
    "hgx_hig_scan_point": (_i, [_vp, _i, _vp, _vp, _vp]),
    "hgx_hig_compute_scan_point": (_i, [_vp, _vp, _i, _i, _vp]),
    "hgx_hig_fit_count": (_i, [_vp, C.POINTER(_i)]),
    "hgx_hig_fit_param": (_i, [_vp, _i, C.c_char_p, C.c_size_t, C.c_char_p, C.c_size_t, _vp, _vp]),
    "hgx_hig_fit_reference": (_i, [_vp, _i, C.c_char_p, C.c_size_t, C.c_char_p, C.c_size_t, _vp, _vp]),
    "hgx_hig_override_qregion": (_i, [_vp, _i, _i, _i]),
    "hgx_hig_fit_algorithm_count": (_i, [_vp, C.POINTER(_i)]),
    "hgx_hig_fit_algorithm": (_i, [_vp, _i, C.c_char_p, C.c_size_t, _vp, _vp, _vp]),
    "hgx_hig_update_param": (_i, [_vp, C.c_char_p, _d]),
    "hgx_hig_fit_update": (_i, [_vp, _vp, _i]),
    "hgx_fit_distance": (_i, [_vp, _i, C.c_long, _vp, _vp, _vp, _vp]),
    "hgx_read_image": (_i, [C.c_char_p, _vp, C.c_long, C.POINTER(C.c_long), C.POINTER(_i), C.POINTER(_i)]),
    "hgx_read_mask": (_i, [C.c_char_p, _vp, C.c_long, C.POINTER(C.c_long)]),
    "hgx_hig_objective": (_i, [_vp, _vp, _vp, _i, _vp, _vp, _i, _d, _vp, C.POINTER(C.c_long)]),
    "hgx_hig_objective_grad": (_i, [_vp, _vp, _vp, _i, _vp, _vp, _i, _d, _vp, _vp]),
    "hgx_hig_population_create": (_i, [_vp, _vp, _i, _vp, _vp, _i, _d, _i, C.POINTER(_vp)]),
    "hgx_hig_population_eval": (_i, [_vp, _vp, _i, _vp]),
    "hgx_hig_population_destroy": (_i, [_vp]),
    "hgx_measure_peaks": (_i, [_vp, _i, C.POINTER(_d), C.POINTER(_d)]),
    "hgx_measure_peak_fp64": (_i, [_vp, C.POINTER(_d)]),
}

_lib = None


class HgxError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"hgx status {status}: {msg}")
        self.status = status


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m hipgisaxs_b200.build`"
                              " (the CUDA library is required; there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def exported_symbols():
    """Names declared in include/hgx.h that the loaded library exports."""
    L = lib()
    return [n for n in SIGNATURES if hasattr(L, n)]


def check(status: int):
    if status != HGX_OK:
        msg = lib().hgx_last_error()
        raise HgxError(status, msg.decode() if msg else "")
    return status
