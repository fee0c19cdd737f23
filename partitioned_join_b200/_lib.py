"""ctypes binding of libpj.so (include/pj.h).  The library is the product:
there is no fallback, a missing or stale build raises at import."""
from __future__ import annotations

import ctypes
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libpj.so")

# status codes (pj_status)
OK, ERR_INVALID, ERR_CAPACITY, ERR_CUDA, ERR_TIMEOUT, ERR_WORKSPACE, ERR_OVERFLOW, ERR_ALIGNMENT, ERR_INTERNAL = range(9)
DIGIT_RAW, DIGIT_HASH = 0, 1
SLOT_FAST, SLOT_REF = 0, 1
SPLIT_HASH, SPLIT_POSITION = 0, 1
TABLE_BUCKET, TABLE_OPEN, TABLE_COMPACT, TABLE_EXACT = 0, 1, 2, 3
NOALLOC_SCRATCH_BYTES = 64 << 20  # PJ_NOALLOC_SCRATCH_BYTES
MAX_HEAVY = 256                   # PJ_MAX_HEAVY
STAGES = ["build_hist", "build_scan", "build_scatter", "build_pass2", "probe_hist", "probe_scan", "probe_scatter",
          "probe_pass2", "join_plan", "join", "total"]


class JoinDesc(ctypes.Structure):
    _fields_ = [("build_keys", ctypes.c_void_p), ("probe_keys", ctypes.c_void_p),
                ("build_payload", ctypes.c_void_p), ("probe_payload", ctypes.c_void_p),
                ("n_build", ctypes.c_int64), ("n_probe", ctypes.c_int64),
                ("key_bytes", ctypes.c_int32), ("payload_bytes", ctypes.c_int32),
                ("unique_build_keys", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class Output(ctypes.Structure):
    _fields_ = [("build_row", ctypes.c_void_p), ("probe_row", ctypes.c_void_p), ("capacity", ctypes.c_int64),
                ("count", ctypes.c_void_p), ("build_payload_out", ctypes.c_void_p),
                ("probe_payload_out", ctypes.c_void_p)]


class Plan(ctypes.Structure):
    _fields_ = [("passes", ctypes.c_int32), ("bits1", ctypes.c_int32), ("bits2", ctypes.c_int32),
                ("digit_mode", ctypes.c_int32), ("table_mode", ctypes.c_int32), ("slot_mode", ctypes.c_int32),
                ("split_mode", ctypes.c_int32), ("table_capacity", ctypes.c_int32), ("probe_chunk", ctypes.c_int32),
                ("wc_tuples", ctypes.c_int32), ("scatter_ctas_per_sm", ctypes.c_int32), ("hist_split", ctypes.c_int32),
                ("max_fill", ctypes.c_float), ("flags", ctypes.c_int32), ("n_heavy", ctypes.c_int32),
                ("heavy_reserved", ctypes.c_int32), ("heavy_keys", ctypes.c_int64 * MAX_HEAVY)]

    def as_dict(self):
        d = {name: getattr(self, name) for name, _ in self._fields_ if name != "heavy_keys"}
        d["heavy_keys"] = list(self.heavy_keys[: max(0, min(self.n_heavy, MAX_HEAVY))])
        return d

    def set_heavy(self, keys):
        keys = list(keys)[:MAX_HEAVY]
        self.n_heavy = len(keys)
        for i, k in enumerate(keys):
            self.heavy_keys[i] = int(k)

    def __repr__(self):
        return "Plan(" + ", ".join(f"{k}={v}" for k, v in self.as_dict().items()) + ")"


class BatchConfig(ctypes.Structure):
    _fields_ = [("direct_threads", ctypes.c_int32), ("direct_chunk", ctypes.c_int32),
                ("direct_max_build", ctypes.c_int32), ("large_bits_delta", ctypes.c_int32),
                ("large_batched", ctypes.c_int32)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class MlpDims(ctypes.Structure):
    _fields_ = [("in_", ctypes.c_int32), ("h1", ctypes.c_int32), ("h2", ctypes.c_int32), ("out", ctypes.c_int32)]


MLP_FEATURES, MLP_HIDDEN, PLAN_CANDIDATES = 32, 64, 30  # PJ_MLP_FEATURES, PJ_MLP_HIDDEN, PJ_PLAN_CANDIDATES
PLAN_CANDIDATE_EXACT = 29  # PJ_PLAN_CANDIDATE_EXACT


# every symbol include/pj.h declares, with its ctypes signature
_P, _I32, _I64, _SZ = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_size_t
SIGNATURES = {
    "pj_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "pj_version": (ctypes.c_char_p, []),
    "pj_plan_default": (ctypes.c_int, [ctypes.POINTER(JoinDesc), ctypes.POINTER(Plan)]),
    "pj_plan_radix": (ctypes.c_int, [ctypes.POINTER(JoinDesc), _I32, _I32, ctypes.c_float, ctypes.POINTER(Plan)]),
    "pj_workspace_size": (ctypes.c_int, [ctypes.POINTER(JoinDesc), ctypes.POINTER(Plan), ctypes.POINTER(_SZ)]),
    "pj_plan_exact": (ctypes.c_int, [ctypes.POINTER(JoinDesc), _P, _SZ, ctypes.POINTER(Plan), _P]),
    "pj_inner_join": (ctypes.c_int, [ctypes.POINTER(JoinDesc), ctypes.POINTER(Plan), ctypes.POINTER(Output), _P, _SZ, _P]),
    "pj_inner_join_timed": (ctypes.c_int, [ctypes.POINTER(JoinDesc), ctypes.POINTER(Plan), ctypes.POINTER(Output), _P, _SZ,
                                           _P, ctypes.POINTER(ctypes.c_float)]),
    "pj_inner_join_events": (ctypes.c_int, [ctypes.POINTER(JoinDesc), ctypes.POINTER(Plan), ctypes.POINTER(Output), _P,
                                            _SZ, _P, ctypes.POINTER(ctypes.c_void_p)]),
    "pj_join_count": (ctypes.c_int, [ctypes.POINTER(JoinDesc), ctypes.POINTER(Plan), _P, _P, _SZ, _P]),
    "pj_check": (ctypes.c_int, [_P, _P]),
    "pj_diag_scan_timeout": (ctypes.c_int, [ctypes.POINTER(JoinDesc), ctypes.POINTER(Plan), _P, _SZ, _I64,
                                            ctypes.c_uint32, _P]),
    "pj_inner_join_noalloc": (ctypes.c_int, [ctypes.POINTER(JoinDesc), ctypes.POINTER(Plan), ctypes.POINTER(Output), _P]),
    "pj_hash_keys": (ctypes.c_int, [_P, _I64, _I32, _P, _P]),
    "pj_hash_slots": (ctypes.c_int, [_P, _I64, _I32, _I32, _I32, _I32, _P, _P]),
    "pj_radix_histogram": (ctypes.c_int, [_P, _I64, _I32, _I32, _I32, _I32, _I32, _P, _P]),
    "pj_partition": (ctypes.c_int, [_P, _I64, _I32, ctypes.POINTER(Plan), _P, _P, _P, _SZ, _P]),
    "pj_partitioned_capacity": (ctypes.c_int, [_I64, _I32, ctypes.POINTER(Plan), ctypes.POINTER(_I64)]),
    "pj_batch_config_default": (ctypes.c_int, [_I32, ctypes.POINTER(BatchConfig)]),
    "pj_batch_workspace_size": (ctypes.c_int, [ctypes.POINTER(JoinDesc), _I32, ctypes.POINTER(BatchConfig),
                                               ctypes.POINTER(_SZ)]),
    "pj_batch_prepare": (ctypes.c_int, [ctypes.POINTER(JoinDesc), ctypes.POINTER(Output), _I32,
                                        ctypes.POINTER(BatchConfig), _P, _SZ, _P]),
    "pj_join_batch": (ctypes.c_int, [ctypes.POINTER(JoinDesc), ctypes.POINTER(Output), _I32,
                                     ctypes.POINTER(BatchConfig), _P, _SZ, _P]),
    "pj_batch_check": (ctypes.c_int, [_P, _P]),
    "pj_batch_autotune": (ctypes.c_int, [ctypes.POINTER(JoinDesc), ctypes.POINTER(Output), _I32, _P, _SZ, _P,
                                         ctypes.POINTER(BatchConfig), ctypes.POINTER(ctypes.c_float)]),
    "pj_mlp_param_count": (ctypes.c_int64, [ctypes.POINTER(MlpDims)]),
    "pj_mlp_forward": (ctypes.c_int, [_P, ctypes.POINTER(MlpDims), _P, _I32, _P, _P, _P]),
    "pj_mlp_backward": (ctypes.c_int, [_P, ctypes.POINTER(MlpDims), _P, _P, _P, _I32, _P, _P, _P]),
    "pj_mlp_mse_grad": (ctypes.c_int, [_P, _P, _P, _I64, _P, _P, _P]),
    "pj_mlp_adam": (ctypes.c_int, [_P, _P, _P, _P, _I64, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                   ctypes.c_float, _I32, _P]),
    "pj_plan_features": (ctypes.c_int, [ctypes.POINTER(JoinDesc), _P, _SZ, ctypes.POINTER(ctypes.c_float),
                                        ctypes.POINTER(Plan), _P]),
    "pj_plan_candidate": (ctypes.c_int, [ctypes.POINTER(JoinDesc), _I32, ctypes.POINTER(Plan), ctypes.POINTER(Plan)]),
    "pj_plan_learned": (ctypes.c_int, [ctypes.POINTER(JoinDesc), _P, _P, _SZ, ctypes.POINTER(Plan),
                                       ctypes.POINTER(ctypes.c_float), _P]),
    "pj_generate_tables": (ctypes.c_int, [_P, _I64, _P, _I64, _I32, _I64, ctypes.c_double, _I32, ctypes.c_double,
                                          ctypes.c_uint64, _P, _P]),
}

_lib = None


def lib():
    """Load libpj.so; raises if the native library has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m partitioned_join_b200.build` "
                               "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


class PJError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        msg = lib().pj_status_string(status).decode()
        super().__init__(f"{what}: {msg} (pj_status {status})" if what else f"{msg} (pj_status {status})")


def check(status: int, what: str = "") -> None:
    if status != OK:
        raise PJError(status, what)
