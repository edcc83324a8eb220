"""ctypes binding of libverona_b200.so (include/verona_b200.h).

The library is built in-tree (verona_b200/build.py). Loading fails loudly if
it is missing: there is no CPU fallback of any kind.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libverona_b200.so")

ABI_VERSION = 1
OK, ERR_ARG, ERR_CUDA, ERR_STATE, ERR_UNSUPPORTED, ERR_NOMEM, ERR_TIMEOUT = 0, -1, -2, -3, -4, -5, -6
RECON = {"minmod": 0, "ppm": 1, "wenoz": 2, "MINMOD": 0, "PPM": 1, "WENOZ": 2}
RIEMANN = {"hll": 0, "hllc": 1, "HLL": 0, "HLLC": 1}
PRECISION = {"fp64": 0, "fp32": 1, "fp32_bulk": 1}
GUESS = {"previous": 0, "learned": 1, "previous_w": 2}
BC_OUTFLOW, BC_FIXED, BC_NOZZLE = 0, 1, 2
FACE = {"xlo": 0, "xhi": 1, "ylo": 2, "yhi": 3, "zlo": 4, "zhi": 5}
CNT_C2P_FAIL, CNT_C2P_FALLBACK, CNT_C2P_ITERS, CNT_C2P_CELLS, CNT_TIMEOUT, CNT_BAD_INDEX, CNT_C2P_FP64 = range(7)
CNT_N = 8


class VBOptions(C.Structure):
    _fields_ = [
        ("version", C.c_uint32),
        ("recon", C.c_int32),
        ("riemann", C.c_int32),
        ("rk", C.c_int32),
        ("precision", C.c_int32),
        ("guess", C.c_int32),
        ("n_iter", C.c_int32),
        ("stats", C.c_int32),
        ("tol", C.c_double),
        ("floor_", C.c_double),
        ("w_rtol", C.c_double),
        ("w_max_newton", C.c_int32),
        ("c2p_fp32", C.c_int32),
        ("reserved_i", C.c_int32 * 6),
        ("reserved_d", C.c_double * 4),
    ]


class VBTuning(C.Structure):
    _fields_ = [("split_con2prim", C.c_int32), ("force_box", C.c_int32), ("learned_fused", C.c_int32),
                ("fp32_pairs", C.c_int32), ("tma_tiles", C.c_int32), ("fp64_contract", C.c_int32),
                ("reserved", C.c_int32 * 2)]


class VBIcParams(C.Structure):
    _fields_ = [("version", C.c_uint32), ("kind", C.c_int32), ("seed", C.c_uint64), ("noise", C.c_double),
                ("rho", C.c_double), ("u", C.c_double), ("box", C.c_double * 3), ("r_max", C.c_double),
                ("r_eng", C.c_double), ("rho0", C.c_double), ("temp", C.c_double), ("outer", C.c_double),
                ("gamma0", C.c_double), ("engine_rho", C.c_double), ("engine_temp", C.c_double),
                ("reserved_d", C.c_double * 4)]


IC_KINDS = {"ambient": 0, "star_jet": 1}


class VBError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"verona_b200 error {code}: {msg}")
        self.code = code


_lib = None
_vp = C.c_void_p
_dp = C.POINTER(C.c_double)

# name -> (argtypes); every function returns int
_SIGS = {
    "vb_default_options": [C.POINTER(VBOptions)],
    "vb_create": [C.POINTER(_vp), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(VBOptions)],
    "vb_destroy": [_vp],
    "vb_set_eos": [_vp, C.c_double],
    "vb_set_grid": [_vp, C.c_double, C.c_double, C.c_double],
    "vb_set_boundary": [_vp, C.c_int, C.c_int, _dp, C.c_int],
    "vb_load_prims": [_vp, _vp, _vp],
    "vb_store_prims": [_vp, _vp, _vp],
    "vb_load_prims_host": [_vp, _vp, _vp],
    "vb_store_prims_host": [_vp, _vp, _vp],
    "vb_store_cons": [_vp, _vp, _vp],
    "vb_default_ic": [C.c_int, C.c_int, C.POINTER(VBIcParams)],
    "vb_init_prims": [_vp, C.POINTER(VBIcParams), _vp],
    "vb_dump_begin": [_vp, _vp, _vp],
    "vb_dump_wait": [_vp, C.POINTER(C.c_uint64)],
    "vb_step": [_vp, C.c_double, C.c_int, _vp],
    "vb_get_time": [_vp, _dp],
    "vb_set_time": [_vp, C.c_double],
    "vb_max_signal_speed": [_vp, _dp, _vp],
    "vb_get_counters": [_vp, C.POINTER(C.c_uint64), C.c_int, _vp],
    "vb_reset_counters": [_vp, _vp],
    "vb_memory_bytes": [_vp, C.POINTER(C.c_uint64)],
    "vb_tma_tiles_active": [_vp, C.POINTER(C.c_int)],
    "vb_profile_enable": [_vp, C.c_int],
    "vb_profile_read": [_vp, _dp, C.POINTER(C.c_int64), C.POINTER(C.c_int64)],
    "vb_profile_read2": [_vp, _dp, _dp, C.POINTER(C.c_int64), C.POINTER(C.c_int64)],
    "vb_set_tuning": [_vp, C.POINTER(VBTuning)],
    "vb_get_tuning": [_vp, C.POINTER(VBTuning)],
    "vb_point_recon": [C.c_int, _vp, _vp, C.c_int, _vp],
    "vb_point_flux": [C.c_int, C.c_int, C.c_int, C.c_double, _vp, _vp, _vp, C.c_int, _vp],
    "vb_point_con2prim": [C.c_int, C.c_double, C.c_int, C.c_double, _vp, _vp, _vp, C.c_int, _vp],
}


def exported_symbols() -> list[str]:
    return list(_SIGS)


def lib():
    """Load the in-tree library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run `python -m verona_b200.build` (no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, args in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_int
        L.vb_last_error.argtypes = [_vp]
        L.vb_last_error.restype = C.c_char_p
        _lib = L
    return _lib


def check(rc: int, handle=None):
    if rc != OK:
        msg = lib().vb_last_error(handle)
        raise VBError(rc, msg.decode() if msg else "")
    return rc


def default_options(**kw) -> VBOptions:
    o = VBOptions()
    check(lib().vb_default_options(C.byref(o)))
    for k, v in kw.items():
        if k == "recon" and isinstance(v, str):
            v = RECON[v]
        elif k == "riemann" and isinstance(v, str):
            v = RIEMANN[v]
        elif k == "precision" and isinstance(v, str):
            v = PRECISION[v]
        elif k == "guess" and isinstance(v, str):
            v = GUESS[v]
        elif k == "floor":
            k = "floor_"
        setattr(o, k, v)
    return o
