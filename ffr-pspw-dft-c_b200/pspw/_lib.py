"""ctypes binding of libpspw_gpu.so (the C ABI in include/pspw_gpu.h).

The library is built in-tree (``ffr-pspw-dft-c_b200/build.py``); there is no
fallback: loading fails loudly when it is missing.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_DIR = os.path.join(PKG_DIR, "lib")
LIB_PATH = os.path.join(LIB_DIR, "libpspw_gpu.so")
DROPIN_PATH = os.path.join(LIB_DIR, "libpspw_dropin.so")

PREC_F64 = 0
PREC_F32 = 1
NL_AUTO = 0
NL_SIMT = 1
NL_TENSOR_CORE = 2
OVERLAP_AUTO = 0
OVERLAP_ON = 1
OVERLAP_OFF = 2
MIX_SIMPLE, MIX_KERKER, MIX_ANDERSON, MIX_PULAY, MIX_BROYDEN = 0, 1, 2, 3, 4

OK = 0
ERRORS = {1: "ARG", 2: "SHAPE", 3: "CUDA", 4: "OOM", 5: "NONFINITE", 6: "TIMEOUT", 7: "LAPACK",
          8: "CHARGE", 9: "NOT_IMPL"}


class PspwError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"pspw error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


class BasisInfo(C.Structure):
    _fields_ = [("nr", C.c_int * 3), ("ngw", C.c_int), ("ngwx", C.c_int), ("ngx", C.c_int),
                ("ng", C.c_int), ("alat", C.c_double), ("omega", C.c_double),
                ("tpiba", C.c_double), ("tpiba2", C.c_double), ("gcut", C.c_double),
                ("gcutw", C.c_double)]


_vp = C.c_void_p
_i = C.c_int
_d = C.c_double

# name -> argtypes (all return int status unless listed in _RESTYPE)
SIGNATURES = {
    "pspw_error_string": [_i],
    "pspw_last_error": [],
    "pspw_version": [],
    "pspw_basis_info_gamma": [_vp, _d, _vp, _vp],
    "pspw_basis_build_gamma": [_vp, _d, _vp, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                               _vp, _vp, _vp, _vp, _vp],
    "pspw_cell_create": [_vp, _i, _i, _i, _i, _i, _i, _vp, _vp, _d, _i, _vp, _i, _vp, _i, _vp,
                         _vp, _vp],
    "pspw_cell_destroy": [_vp],
    "pspw_cell_set_veff": [_vp, _vp, _i],
    "pspw_cell_set_veff_device": [_vp, _vp, _i],
    "pspw_cell_get_stream": [_vp, _vp],
    "pspw_cell_synchronize": [_vp],
    "pspw_cell_sizes": [_vp, _vp],
    "pspw_cell_set_band_batch": [_vp, _i],
    "pspw_cell_set_nl_path": [_vp, _i],
    "pspw_cell_set_nl_overlap": [_vp, _i],
    "pspw_cell_check_device_wait": [_vp, _i],
    "pspw_apply_ham_block": [_vp, _vp, _vp, _i, _i],
    "pspw_apply_ham_block_dev": [_vp, _i, _vp, _vp, _i, _i, _i],
    "pspw_apply_ham_block_dev_noalloc": [_vp, _i, _vp, _vp, _i, _i, _i],
    "pspw_chebyfilt": [_vp, _vp, _i, _i, _i, _d, _d, _i],
    "pspw_chebyfilt_dev": [_vp, _i, _vp, _i, _i, _i, _i, _d, _d],
    "pspw_timing_enable": [_vp, _i],
    "pspw_timing_read": [_vp, _i, _vp, _vp],
    "pspw_timing_reset": [_vp],
    "pspw_kernel_launches": [_vp, _vp],
    "pspw_random_col": [_vp, _i, C.c_long],
    "pspw_gen_prec": [_vp, _vp, _i, _d],
    "pspw_ortho_qr": [_vp, _vp, _i, _i],
    "pspw_eig_zheevd": [_vp, _vp, _i, _vp, _i],
    "pspw_eig_zhegv": [_vp, _vp, _i, _vp, _i, _vp, _i, _i],
    "pspw_eig_zhegv_eval": [_vp, _vp, _i, _vp, _i, _vp, _vp, _i, _i],
    "pspw_davidson": [_vp, _vp, _vp, _i, _i, _vp, _i, _i, _i, _vp, _vp],
    "pspw_lobpcg": [_vp, _vp, _vp, _i, _i, _vp, _i, _i, _i, _vp, _vp],
    "pspw_lobpcg_ortho": [_vp, _vp, _vp, _i, _i, _vp, _i, _i, _i, _vp, _vp],
    "pspw_lobpcg_ortho_from": [_vp, _vp, _vp, _i, _i, _vp, _i, _i, _i, _vp, _vp],
    "pspw_lanczos": [_vp, _vp, _i, _i, _vp, _i, _vp],
    "pspw_eval_rho_psi": [_vp, _vp, _vp, _i, _i, _i, _vp, _d, _d, _vp],
    "pspw_eval_enl": [_vp, _vp, _i, _i, _i, _vp, _d, _vp, _vp],
    "pspw_eval_rho_psi_dev": [_vp, _vp, _vp, _i, _i, _i, _vp, _d, _d, _vp],
    "pspw_eval_enl_dev": [_vp, _vp, _i, _i, _i, _vp, _d, _vp, _vp],
    "pspw_scf_create": [_vp, _i, _vp, _vp, _vp, _vp, _i, _vp, _vp, _vp, _d, _d, _d, _d, _vp],
    "pspw_scf_destroy": [_vp],
    "pspw_eval_energy": [_vp, _vp, _d, _d, _vp],
    "pspw_eval_energy_dev": [_vp, _vp, _d, _d, _vp],
    "pspw_xc_pz": [_vp, _vp, _vp, _vp],
    "pspw_normalize_rho": [_vp, _vp, _vp],
    "pspw_kerker_prec": [_vp, _vp, _d, _d],
    "pspw_xc_pz_dev": [_vp, _vp, _vp, _vp],
    "pspw_normalize_rho_dev": [_vp, _vp, _vp],
    "pspw_kerker_prec_dev": [_vp, _vp, _d, _d],
    "pspw_mix_init": [_vp, _i, _i, _d, _d, _vp],
    "pspw_mix": [_vp, _i, _vp, _vp],
    "pspw_mix_dev": [_vp, _i, _vp, _vp],
    "pspw_cheby_scf": [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "pspw_system_load": [C.c_char_p, _i, _vp],
    "pspw_system_destroy": [_vp],
    "pspw_system_info": [_vp, _vp, _vp],
    "pspw_system_params": [_vp, _vp],
    "pspw_system_array": [_vp, _i, _vp, C.c_longlong],
    "pspw_system_cell": [_vp, _vp],
    "pspw_system_scf": [_vp, _vp],
    "pspw_system_timing": [_vp, _vp],
    "pspw_system_cheby_scf": [_vp, _i, C.c_char_p, _vp, _vp, _vp, _vp, _vp],
    "pspw_system_cheby_scf_with": [_vp, _vp, C.c_char_p, _vp, _vp, _vp, _vp, _vp],
    "pspw_print_3d_array": [_vp, _i, _i, _i, C.c_char_p],
    "pspw_system_species": [_vp, _vp, _vp],
    "pspw_batch_create": [_i, _vp, _vp, _i, _vp],
    "pspw_batch_blocks": [_vp, _i, _vp, _vp],
    "pspw_batch_upload": [_vp, _i, _vp],
    "pspw_batch_download": [_vp, _i, _vp],
    "pspw_batch_tune": [_vp, _i],
    "pspw_batch_schedule": [_vp, _i, _vp, _vp, _vp],
    "pspw_batch_apply": [_vp],
    "pspw_batch_kernels": [_vp, _vp],
    "pspw_batch_stream": [_vp, _vp],
    "pspw_batch_synchronize": [_vp],
    "pspw_batch_destroy": [_vp],
    "pspw_server_create": [_i, _vp, _vp],
    "pspw_server_submit": [_vp, C.c_char_p, _vp],
    "pspw_server_wait": [_vp, _i, _vp, _vp, _i],
    "pspw_server_now": [_vp, _vp],
    "pspw_server_destroy": [_vp],
    "pspw_zgemm_dev": [_vp, C.c_char, _i, _i, _i, _vp, _vp, _i, _vp, _i, _vp, _vp, _i],
    "pspw_eig_zheevd_dev": [_vp, _vp, _i, _vp, _i],
    "pspw_ortho_span_dev": [_vp, _vp, _i, _i],
}
_RESTYPE = {"pspw_error_string": C.c_char_p, "pspw_last_error": C.c_char_p}

_LIB = None


def lib():
    """Load libpspw_gpu.so once (raises if it was not built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python ffr-pspw-dft-c_b200/build.py`")
        L = C.CDLL(LIB_PATH, mode=C.RTLD_GLOBAL)
        for name, args in SIGNATURES.items():
            f = getattr(L, name, None)
            if f is None:
                continue
            f.argtypes = args
            f.restype = _RESTYPE.get(name, C.c_int)
        _LIB = L
    return _LIB


def check(rc):
    if rc != OK:
        msg = lib().pspw_last_error()
        raise PspwError(rc, msg.decode() if msg else "")
    return rc


def ptr(a):
    """Address of a numpy array or a torch tensor (device or host)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()
