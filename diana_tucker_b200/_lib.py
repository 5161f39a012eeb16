"""ctypes binding of libdt_cuda.so (the C ABI declared in include/dt_cuda.h).

The library is built in-tree by ``diana_tucker_b200.build``; importing this
module never falls back to anything else: a missing or unloadable library
raises immediately.
"""
from __future__ import annotations

import ctypes
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libdt_cuda.so")

DT_OK = 0
DT_ERR_ARG = 1
DT_ERR_CUDA = 2
DT_ERR_NOMEM = 3
DT_ERR_NUMERIC = 4
DT_ERR_UNSUPPORTED = 5
DT_ERR_TIMEOUT = 6

DT_F64 = 0
DT_F32 = 1

DT_INIT_RANDN_LIBC = 0
DT_INIT_HOSVD = 1
DT_INIT_GIVEN = 2

DT_PREC_FP64 = 0
DT_PREC_BF16 = 1
DT_PREC_BF16X2 = 2
DT_PREC_BF16XH = 3

DT_MAX_HIST = 256

c_dp = ctypes.POINTER(ctypes.c_double)
c_i64p = ctypes.POINTER(ctypes.c_int64)


class HooiOpts(ctypes.Structure):
    _fields_ = [
        ("init", ctypes.c_int),
        ("seed", ctypes.c_uint),
        ("max_sweeps", ctypes.c_int),
        ("tol", ctypes.c_double),
        ("inner_iters", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("refine_sweeps", ctypes.c_int),
        ("verbose", ctypes.c_int),
        ("profile", ctypes.c_int),
    ]


class HooiReport(ctypes.Structure):
    _fields_ = [
        ("sweeps", ctypes.c_int),
        ("x_norm", ctypes.c_double),
        ("g_norm", ctypes.c_double),
        ("residual", ctypes.c_double),
        ("device_ms", ctypes.c_double),
        ("res_hist", ctypes.c_double * DT_MAX_HIST),
        ("kernel_launches", ctypes.c_int),
        ("precision_used", ctypes.c_int),
        ("ttm_x_launches", ctypes.c_int),
        ("ttm_x_ms", ctypes.c_double),
        ("ttm_x_bytes", ctypes.c_double),
    ]

    def as_dict(self):
        return {
            "sweeps": self.sweeps,
            "x_norm": self.x_norm,
            "g_norm": self.g_norm,
            "residual": self.residual,
            "device_ms": self.device_ms,
            "res_hist": list(self.res_hist[: min(self.sweeps, DT_MAX_HIST)]),
            "kernel_launches": self.kernel_launches,
            "precision_used": self.precision_used,
            "ttm_x_launches": self.ttm_x_launches,
            "ttm_x_ms": self.ttm_x_ms,
            "ttm_x_bytes": self.ttm_x_bytes,
        }


class BatchedReport(ctypes.Structure):
    _fields_ = [
        ("device_ms", ctypes.c_double),
        ("block_threads", ctypes.c_int),
        ("grid", ctypes.c_int),
        ("kernel_launches", ctypes.c_int),
        ("pack", ctypes.c_int),
        ("items", ctypes.c_int),
        ("candidates_timed", ctypes.c_int),
        ("tune_best_ms", ctypes.c_double),
        ("tune_worst_ms", ctypes.c_double),
        ("graph_reused", ctypes.c_int),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


# (name, restype, argtypes)
_vp = ctypes.c_void_p
_SIGS = [
    ("dt_ctx_create", ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_vp)]),
    ("dt_ctx_destroy", ctypes.c_int, [_vp]),
    ("dt_ctx_set_stream", ctypes.c_int, [_vp, _vp]),
    ("dt_ctx_synchronize", ctypes.c_int, [_vp]),
    ("dt_last_error", ctypes.c_char_p, []),
    ("dt_ctx_kernel_launches", ctypes.c_int64, [_vp]),
    ("dt_ctx_set_mem_limit", ctypes.c_int, [_vp, ctypes.c_uint64]),
    ("dt_ctx_mem_usage", ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_uint64),
                                        ctypes.POINTER(ctypes.c_uint64)]),
    ("dt_selftest_wait_timeout", ctypes.c_int, [_vp, ctypes.c_int64]),
    ("dt_libc_rand_sequence", ctypes.c_int, [ctypes.c_uint, ctypes.c_int64, _vp]),
    ("dt_ttm_f64", ctypes.c_int, [_vp, _vp, ctypes.c_int, c_i64p, ctypes.c_int, _vp,
                                  ctypes.c_int64, _vp]),
    ("dt_gram_f64", ctypes.c_int, [_vp, _vp, ctypes.c_int, c_i64p, ctypes.c_int, _vp]),
    ("dt_ws_loss_grad", ctypes.c_int, [_vp, _vp, ctypes.c_int64, ctypes.c_int64, ctypes.c_int,
                                       _vp, _vp, _vp, _vp, _vp]),
    ("dt_ws_train", ctypes.c_int, [_vp, _vp, ctypes.c_int64, ctypes.c_int64, ctypes.c_int,
                                   ctypes.c_int, ctypes.c_double, ctypes.c_uint64, _vp, _vp, _vp]),
    ("dt_ws_init", ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_int, c_i64p, c_i64p, _vp,
                                  ctypes.c_int, ctypes.c_int, _vp, c_dp, c_dp]),
    ("dt_gram_f64_noalloc", ctypes.c_int, [_vp, _vp, ctypes.c_int, c_i64p, ctypes.c_int,
                                           _vp]),
    ("dt_ttt_except_f64", ctypes.c_int, [_vp, _vp, c_i64p, _vp, c_i64p, ctypes.c_int,
                                         ctypes.c_int, _vp]),
    ("dt_fnorm_f64", ctypes.c_int, [_vp, _vp, ctypes.c_int64, c_dp]),
    ("dt_matmul_f64", ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int64,
                                     ctypes.c_int64, ctypes.c_int64, _vp, _vp, _vp]),
    ("dt_reduced_qr_f64", ctypes.c_int, [_vp, _vp, ctypes.c_int64, ctypes.c_int64, _vp, _vp]),
    ("dt_inverse_f64", ctypes.c_int, [_vp, _vp, ctypes.c_int64, _vp]),
    ("dt_orth2_f64", ctypes.c_int, [_vp, _vp, ctypes.c_int64, ctypes.c_int64]),
    ("dt_als_f64", ctypes.c_int, [_vp, _vp, ctypes.c_int, c_i64p, ctypes.c_int, _vp,
                                  ctypes.c_int64, ctypes.c_int, _vp]),
    ("dt_ttm_tc", ctypes.c_int, [_vp, _vp, ctypes.c_int, c_i64p, ctypes.c_int, _vp,
                                 ctypes.c_int64, ctypes.c_int, _vp]),
    ("dt_gram_tc", ctypes.c_int, [_vp, _vp, ctypes.c_int64, ctypes.c_int64, ctypes.c_int, _vp]),
    ("dt_hooi_dense", ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_int, c_i64p, c_i64p,
                                     ctypes.POINTER(HooiOpts), _vp, ctypes.POINTER(_vp),
                                     ctypes.POINTER(HooiReport)]),
    ("dt_hooi_default_opts", None, [ctypes.POINTER(HooiOpts)]),
    ("dt_hooi_batched", ctypes.c_int, [_vp, ctypes.c_int, c_i64p, c_i64p, _vp, c_i64p,
                                       ctypes.c_int, ctypes.c_int, _vp, c_i64p, _vp, c_i64p,
                                       _vp, ctypes.c_int, ctypes.POINTER(BatchedReport)]),
    ("dt_sptensor_create", ctypes.c_int, [_vp, ctypes.c_int64, ctypes.c_int,
                                          ctypes.POINTER(_vp), _vp, c_i64p,
                                          ctypes.POINTER(_vp)]),
    ("dt_sptensor_destroy", ctypes.c_int, [_vp]),
    ("dt_sp_fnorm", ctypes.c_int, [_vp, _vp, c_dp]),
    ("dt_sp_ttmc_mTR", ctypes.c_int, [_vp, _vp, ctypes.POINTER(_vp), c_i64p, ctypes.c_int,
                                      _vp]),
    ("dt_sp_ttmc_mTL", ctypes.c_int, [_vp, _vp, ctypes.POINTER(_vp), c_i64p, ctypes.c_int,
                                      _vp, _vp]),
    ("dt_sp_ttmc_rows", ctypes.c_int, [_vp, _vp, ctypes.POINTER(_vp), c_i64p, ctypes.c_int,
                                       _vp]),
    ("dt_sp_hooi", ctypes.c_int, [_vp, _vp, c_i64p, ctypes.c_int, ctypes.POINTER(_vp), _vp,
                                  ctypes.POINTER(HooiReport)]),
    ("dt_sp_ttmc_dense_f64", ctypes.c_int, [_vp, _vp, ctypes.POINTER(_vp), c_i64p,
                                            ctypes.POINTER(ctypes.c_int), ctypes.c_int, _vp]),
    ("dt_sp_mettmc_f64", ctypes.c_int, [_vp, _vp, ctypes.POINTER(_vp), c_i64p,
                                        ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_int,
                                        _vp]),
    ("dt_tns_read", ctypes.c_int, [_vp, ctypes.c_char_p, ctypes.POINTER(_vp),
                                   ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int64)]),
    ("dt_tns_parse", ctypes.c_int, [_vp, _vp, ctypes.c_int64, ctypes.POINTER(_vp),
                                    ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int64)]),
    ("dt_tns_copy", ctypes.c_int, [_vp, _vp, c_i64p, ctypes.POINTER(_vp), _vp]),
    ("dt_tns_to_sptensor", ctypes.c_int, [_vp, _vp, ctypes.POINTER(_vp)]),
    ("dt_tns_destroy", ctypes.c_int, [_vp]),
    ("dt_summary_enable", ctypes.c_int, [_vp, ctypes.c_int]),
    ("dt_summary_reset", ctypes.c_int, [_vp]),
    ("dt_summary_table", ctypes.c_int, [_vp, ctypes.c_char_p, ctypes.c_int64,
                                        ctypes.POINTER(ctypes.c_int64)]),
]

EXPORTED = [s[0] for s in _SIGS]

_lib = None


def load(path: str = LIB_PATH):
    """Loads libdt_cuda.so and declares every signature; raises if absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(
            f"libdt_cuda.so not built ({path}); run `python -m diana_tucker_b200.build`")
    lib = ctypes.CDLL(path)
    for name, res, args in _SIGS:
        fn = getattr(lib, name)  # AttributeError if a declared symbol is missing
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class DTError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[dt error {code}] {msg}")
        self.code = code


def check(code: int):
    if code != DT_OK:
        msg = _lib.dt_last_error().decode(errors="replace") if _lib else ""
        raise DTError(code, msg)
