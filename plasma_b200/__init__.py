"""plasma_b200 -- B200-native implementation of PLASMA's SPD path.

The product is the C-ABI shared library ``libplasma_b200.so`` next to this
file (built from ``csrc/`` by ``make -C plasma_b200/csrc``); its interface is
the PLASMA C API declared in ``include/*.h``.  This module binds that library
with ctypes so Python callers (tests, benchmarks, the autograd binding) go
through exactly the entry points a C caller uses.

Matrices cross the boundary as column-major arrays, as in the reference's
LAPACK-layout routines (compute/zpotrf.c:74-150 and siblings): a host numpy
array in Fortran order, or a device buffer given by pointer.  torch is used
only to own device memory.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import (POINTER, Structure, byref, c_double, c_float, c_int,
                    c_longlong, c_size_t, c_void_p, c_char_p)

# The library keeps about 16 CUDA streams busy while a host matrix is still
# being uploaded; more hardware queues than the driver's default 8 keep them
# from holding one another up.  The driver reads this when the CUDA context
# is created, so it is set at import, before torch touches the GPU.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libplasma_b200.so")

# ---------------------------------------------------------------------------
# constants (include/plasma_types.h; values equal the reference's)
# ---------------------------------------------------------------------------
PlasmaRealFloat = 2
PlasmaRealDouble = 3
PlasmaNoTrans = 111
PlasmaTrans = 112
PlasmaUpper = 121
PlasmaLower = 122
PlasmaGeneral = 123
PlasmaGeneralBand = 124
PlasmaSuccess = 0
PlasmaErrorNotInitialized = -101
PlasmaErrorNotSupported = -102
PlasmaErrorIllegalValue = -103
PlasmaErrorOutOfMemory = -104
PlasmaErrorEnvironment = -109
PlasmaDisabled = 0
PlasmaEnabled = 1
PlasmaTuning = 0
PlasmaNb = 1
PlasmaIb = 2
PlasmaMixedPrecisionMode = 1000
PlasmaRefinement = 1001
PlasmaDevice = 1002
PlasmaLookahead = 1003
PlasmaFactorFP32 = 0
PlasmaFactorTF32 = 1
PlasmaFactorBF16 = 2
PlasmaFactorAuto = 3
PlasmaRefineIR = 0
PlasmaRefineGMRES = 1
PlasmaRefineAuto = 2


class plasma_desc_t(Structure):
    """Mirror of the descriptor struct of include/plasma_descriptor.h."""
    _fields_ = [
        ("type", c_int), ("uplo", c_int), ("precision", c_int),
        ("matrix", c_void_p), ("A21", c_size_t), ("A12", c_size_t),
        ("A22", c_size_t),
        ("mb", c_int), ("nb", c_int),
        ("gm", c_int), ("gn", c_int), ("gmt", c_int), ("gnt", c_int),
        ("i", c_int), ("j", c_int), ("m", c_int), ("n", c_int),
        ("mt", c_int), ("nt", c_int),
        ("kl", c_int), ("ku", c_int), ("klt", c_int), ("kut", c_int),
    ]


class plasma_request_t(Structure):
    _fields_ = [("status", c_int)]


class plasma_sequence_t(Structure):
    _fields_ = [("status", c_int), ("request", POINTER(plasma_request_t))]


class plasma_dsposv_info_t(Structure):
    _fields_ = [
        ("factor_mode", c_int), ("refinement", c_int),
        ("ir_iterations", c_int), ("gmres_iterations", c_int),
        ("fallback_fp64", c_int), ("attempts", c_int),
        ("backward_error", c_double), ("anorm", c_double),
        ("factor_ms", c_double), ("refine_ms", c_double),
    ]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


_lib = None

# (name, restype, argtypes) of every exported entry point
_D = POINTER(c_double)
_S = POINTER(c_float)
_DESC = plasma_desc_t
_SEQ = POINTER(plasma_sequence_t)
_REQ = POINTER(plasma_request_t)
_SIGNATURES = [
    ("plasma_init", c_int, []),
    ("plasma_finalize", c_int, []),
    ("plasma_set", c_int, [c_int, c_int]),
    ("plasma_get", c_int, [c_int, POINTER(c_int)]),
    ("plasma_version", None, [POINTER(c_int)] * 3),
    ("plasma_dpotrf", c_int, [c_int, c_int, c_void_p, c_int]),
    ("plasma_spotrf", c_int, [c_int, c_int, c_void_p, c_int]),
    ("plasma_dpotrs", c_int, [c_int, c_int, c_int, c_void_p, c_int, c_void_p, c_int]),
    ("plasma_spotrs", c_int, [c_int, c_int, c_int, c_void_p, c_int, c_void_p, c_int]),
    ("plasma_dposv", c_int, [c_int, c_int, c_int, c_void_p, c_int, c_void_p, c_int]),
    ("plasma_sposv", c_int, [c_int, c_int, c_int, c_void_p, c_int, c_void_p, c_int]),
    ("plasma_dsposv", c_int, [c_int, c_int, c_int, c_void_p, c_int, c_void_p,
                              c_int, c_void_p, c_int, POINTER(c_int)]),
    ("plasma_dsposv_ex", c_int, [c_int, c_int, c_int, c_void_p, c_int, c_void_p,
                                 c_int, c_void_p, c_int, POINTER(c_int),
                                 POINTER(plasma_dsposv_info_t)]),
    ("plasma_omp_dpotrf", None, [c_int, _DESC, _SEQ, _REQ]),
    ("plasma_omp_spotrf", None, [c_int, _DESC, _SEQ, _REQ]),
    ("plasma_omp_dpotrs", None, [c_int, _DESC, _DESC, _SEQ, _REQ]),
    ("plasma_omp_dpotrs_noalloc", None, [c_int, _DESC, _DESC, _SEQ, _REQ]),
    ("plasma_batch_create", c_int, [c_int, c_int, c_void_p, POINTER(c_void_p)]),
    ("plasma_batch_destroy", None, [c_void_p]),
    ("plasma_batch_matrix_elems", c_longlong, [c_void_p]),
    ("plasma_batch_vector_elems", c_longlong, [c_void_p]),
    ("plasma_batch_offsets", c_int, [c_void_p, c_void_p, c_void_p]),
    ("plasma_batch_set_graph", c_int, [c_void_p, c_int]),
    ("plasma_dposv_batched", c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    ("plasma_sposv_batched", c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    ("plasma_dpotrf_batched", c_int, [c_void_p, c_void_p, c_void_p]),
    ("plasma_spotrf_batched", c_int, [c_void_p, c_void_p, c_void_p]),
    ("plasma_dpotrs_batched", c_int, [c_void_p, c_void_p, c_void_p]),
    ("plasma_spotrs_batched", c_int, [c_void_p, c_void_p, c_void_p]),
    ("plasma_dpotrf_adjoint_batched", c_int, [c_void_p, c_void_p, c_void_p]),
    ("plasma_spotrf_adjoint_batched", c_int, [c_void_p, c_void_p, c_void_p]),
    ("plasma_dpotrs_adjoint_batched", c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    ("plasma_spotrs_adjoint_batched", c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    ("plasma_tuning_get_batched_nb", c_int, [c_int, c_int]),
    ("plasma_autotune_potrf", c_int, [c_int, c_int, POINTER(c_double)]),
    ("plasma_autotune_batched", c_int, [c_int, c_int]),
    ("plasma_tuning_set_batched_nb", c_int, [c_int, c_int, c_int]),
    ("plasma_dpotrf_adjoint", c_int, [c_int, c_int, c_void_p, c_int, c_void_p, c_int]),
    ("plasma_spotrf_adjoint", c_int, [c_int, c_int, c_void_p, c_int, c_void_p, c_int]),
    ("plasma_dpotrs_adjoint", c_int, [c_int, c_int, c_int, c_void_p, c_int, c_void_p,
                                      c_int, c_void_p, c_int, c_void_p, c_int]),
    ("plasma_spotrs_adjoint", c_int, [c_int, c_int, c_int, c_void_p, c_int, c_void_p,
                                      c_int, c_void_p, c_int, c_void_p, c_int]),
    ("plasma_omp_dpotrf_adjoint", None, [c_int, _DESC, _DESC, _SEQ, _REQ]),
    ("plasma_omp_spotrf_adjoint", None, [c_int, _DESC, _DESC, _SEQ, _REQ]),
    ("plasma_omp_dpotrs_adjoint", None, [c_int, _DESC, _DESC, _DESC, _DESC, _SEQ, _REQ]),
    ("plasma_omp_spotrs_adjoint", None, [c_int, _DESC, _DESC, _DESC, _DESC, _SEQ, _REQ]),
    ("plasma_omp_spotrs", None, [c_int, _DESC, _DESC, _SEQ, _REQ]),
    ("plasma_dpotri", c_int, [c_int, c_int, c_void_p, c_int]),
    ("plasma_spotri", c_int, [c_int, c_int, c_void_p, c_int]),
    ("plasma_dpoinv", c_int, [c_int, c_int, c_void_p, c_int]),
    ("plasma_spoinv", c_int, [c_int, c_int, c_void_p, c_int]),
    ("plasma_omp_dpotri", None, [c_int, _DESC, _SEQ, _REQ]),
    ("plasma_omp_spotri", None, [c_int, _DESC, _SEQ, _REQ]),
    ("plasma_omp_dpoinv", None, [c_int, _DESC, _SEQ, _REQ]),
    ("plasma_omp_spoinv", None, [c_int, _DESC, _SEQ, _REQ]),
    ("plasma_dpbtrf", c_int, [c_int, c_int, c_int, c_void_p, c_int]),
    ("plasma_spbtrf", c_int, [c_int, c_int, c_int, c_void_p, c_int]),
    ("plasma_dpbtrs", c_int, [c_int, c_int, c_int, c_int, c_void_p, c_int, c_void_p, c_int]),
    ("plasma_spbtrs", c_int, [c_int, c_int, c_int, c_int, c_void_p, c_int, c_void_p, c_int]),
    ("plasma_dpbsv", c_int, [c_int, c_int, c_int, c_int, c_void_p, c_int, c_void_p, c_int]),
    ("plasma_spbsv", c_int, [c_int, c_int, c_int, c_int, c_void_p, c_int, c_void_p, c_int]),
    ("plasma_omp_dpbtrf", None, [c_int, _DESC, _SEQ, _REQ]),
    ("plasma_omp_spbtrf", None, [c_int, _DESC, _SEQ, _REQ]),
    ("plasma_omp_dpbtrs", None, [c_int, _DESC, _DESC, _SEQ, _REQ]),
    ("plasma_omp_spbtrs", None, [c_int, _DESC, _DESC, _SEQ, _REQ]),
    ("plasma_omp_dpbsv", None, [c_int, _DESC, _DESC, _SEQ, _REQ]),
    ("plasma_omp_spbsv", None, [c_int, _DESC, _DESC, _SEQ, _REQ]),
    ("plasma_omp_dpb2desc", None, [c_void_p, c_int, _DESC, _SEQ, _REQ]),
    ("plasma_omp_spb2desc", None, [c_void_p, c_int, _DESC, _SEQ, _REQ]),
    ("plasma_omp_ddesc2pb", None, [_DESC, c_void_p, c_int, _SEQ, _REQ]),
    ("plasma_omp_sdesc2pb", None, [_DESC, c_void_p, c_int, _SEQ, _REQ]),
    ("plasma_omp_dposv", None, [c_int, _DESC, _DESC, _SEQ, _REQ]),
    ("plasma_omp_sposv", None, [c_int, _DESC, _DESC, _SEQ, _REQ]),
    ("plasma_dsgesv", c_int, [c_int, c_int, c_void_p, c_int, c_void_p, c_void_p, c_int,
                              c_void_p, c_int, POINTER(c_int)]),
    ("plasma_omp_dsgesv", None, [_DESC, c_void_p, _DESC, _DESC, _DESC, _DESC, _DESC,
                                 c_void_p, c_void_p, c_void_p, POINTER(c_int), _SEQ, _REQ]),
    ("plasma_omp_dsposv", None, [c_int, _DESC, _DESC, _DESC, _DESC, _DESC, _DESC,
                                 c_void_p, c_void_p, c_void_p, POINTER(c_int),
                                 _SEQ, _REQ]),
    ("plasma_omp_dge2desc", None, [c_void_p, c_int, _DESC, _SEQ, _REQ]),
    ("plasma_omp_ddesc2ge", None, [_DESC, c_void_p, c_int, _SEQ, _REQ]),
    ("plasma_omp_dtr2desc", None, [c_void_p, c_int, _DESC, _SEQ, _REQ]),
    ("plasma_omp_ddesc2tr", None, [_DESC, c_void_p, c_int, _SEQ, _REQ]),
    ("plasma_omp_sge2desc", None, [c_void_p, c_int, _DESC, _SEQ, _REQ]),
    ("plasma_omp_sdesc2ge", None, [_DESC, c_void_p, c_int, _SEQ, _REQ]),
    ("plasma_omp_str2desc", None, [c_void_p, c_int, _DESC, _SEQ, _REQ]),
    ("plasma_omp_sdesc2tr", None, [_DESC, c_void_p, c_int, _SEQ, _REQ]),
    ("plasma_desc_general_create", c_int, [c_int] * 9 + [POINTER(plasma_desc_t)]),
    ("plasma_desc_triangular_create", c_int, [c_int] * 10 + [POINTER(plasma_desc_t)]),
    ("plasma_desc_destroy", c_int, [POINTER(plasma_desc_t)]),
    ("plasma_desc_general_init", c_int, [c_int, c_void_p] + [c_int] * 8
     + [POINTER(plasma_desc_t)]),
    ("plasma_desc_triangular_init", c_int, [c_int, c_int, c_void_p] + [c_int] * 8
     + [POINTER(plasma_desc_t)]),
    ("plasma_desc_general_band_create", c_int, [c_int] * 12 + [POINTER(plasma_desc_t)]),
    ("plasma_desc_general_band_init", c_int, [c_int, c_int, c_void_p] + [c_int] * 10
     + [POINTER(plasma_desc_t)]),
    ("plasma_desc_check", c_int, [_DESC]),
    ("plasma_desc_general_band_check", c_int, [_DESC]),
    ("plasma_desc_general_check", c_int, [_DESC]),
    ("plasma_desc_view", plasma_desc_t, [_DESC, c_int, c_int, c_int, c_int]),
    ("plasma_desc_storage_bytes", c_size_t, [_DESC]),
    ("plasma_request_fail", c_int, [_SEQ, _REQ, c_int]),
    ("plasma_request_init", c_int, [_REQ]),
    ("plasma_sequence_init", c_int, [_SEQ]),
    ("plasma_sequence_wait", c_int, [_SEQ]),
    ("plasma_set_stream", c_int, [c_void_p]),
    ("plasma_get_stream", c_void_p, []),
    ("plasma_kernel_launches", c_longlong, []),
    ("plasma_device_allocations", c_longlong, []),
    ("plasma_strerror", c_char_p, [c_int]),
    ("plasma_profile_enable", None, [c_int]),
    ("plasma_profile_query", c_int, [c_int, POINTER(c_longlong), POINTER(c_double),
                                     POINTER(c_double), POINTER(c_double)]),
    ("plasma_tuning_get_potrf_nb", c_int, [c_int, c_int]),
    ("plasma_tuning_set_potrf_nb", c_int, [c_int, c_int, c_int]),
    ("plasma_uplo_const", c_int, [ctypes.c_char]),
    ("plasma_trans_const", c_int, [ctypes.c_char]),
    ("plasma_side_const", c_int, [ctypes.c_char]),
    ("plasma_diag_const", c_int, [ctypes.c_char]),
    ("plasma_norm_const", c_int, [ctypes.c_char]),
]


def lib():
    """Loads libplasma_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `make -C plasma_b200/csrc` "
                "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in _SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def exported_symbols():
    return [s[0] for s in _SIGNATURES]


# ---------------------------------------------------------------------------
# thin helpers
# ---------------------------------------------------------------------------
def init(device: int | None = None) -> int:
    L = lib()
    if device is not None:
        L.plasma_set(PlasmaDevice, device)
    return L.plasma_init()


def finalize() -> int:
    return lib().plasma_finalize()


def set_param(param: int, value: int) -> int:
    return lib().plasma_set(param, value)


def get_param(param: int) -> int:
    v = c_int(0)
    rc = lib().plasma_get(param, byref(v))
    if rc != 0:
        raise RuntimeError(f"plasma_get({param}) -> {rc}")
    return v.value


def new_sequence():
    seq, req = plasma_sequence_t(), plasma_request_t()
    lib().plasma_sequence_init(byref(seq))
    lib().plasma_request_init(byref(req))
    return seq, req


def ptr(x) -> int:
    """Raw address of a numpy array or torch tensor."""
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    return x.ctypes.data


def launches() -> int:
    return lib().plasma_kernel_launches()


KCLASS = {"potrf": 0, "trsm": 1, "update": 2, "solve": 3, "aux": 4}


def profile_enable(on: bool = True) -> None:
    lib().plasma_profile_enable(1 if on else 0)


def profile_query(kclass: str) -> dict:
    n, ms, fl, by = c_longlong(), c_double(), c_double(), c_double()
    lib().plasma_profile_query(KCLASS[kclass], byref(n), byref(ms), byref(fl), byref(by))
    return {"launches": n.value, "ms": ms.value, "flops": fl.value, "bytes": by.value}
