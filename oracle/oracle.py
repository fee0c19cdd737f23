"""ctypes front end of the oracle (oracle/pj_oracle.c -> oracle/libpj_oracle.so)
and of the reference's own code compiled into oracle/_ref/.

TEST INFRASTRUCTURE ONLY.  Functions cite the reference lines they restate
in oracle/pj_oracle.c.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libpj_oracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_lib = None


def build_oracle() -> None:
    """Compile oracle/pj_oracle.c (gcc) into oracle/libpj_oracle.so."""
    src = os.path.join(HERE, "pj_oracle.c")
    subprocess.check_call(["gcc", "-O2", "-std=c99", "-fPIC", "-shared", src, "-o", ORACLE_SO])


def lib():
    global _lib
    if _lib is None:
        src = os.path.join(HERE, "pj_oracle.c")
        if not os.path.exists(ORACLE_SO) or os.path.getmtime(ORACLE_SO) < os.path.getmtime(src):
            build_oracle()
        L = ctypes.CDLL(ORACLE_SO)
        P, I64, I32, U32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_uint32
        L.pjo_hash_i32.restype, L.pjo_hash_i32.argtypes = U32, [I32]
        L.pjo_hash_i64.restype, L.pjo_hash_i64.argtypes = U32, [I64]
        L.pjo_hash_array.restype, L.pjo_hash_array.argtypes = None, [P, I64, ctypes.c_int, P]
        L.pjo_ref_slot.restype, L.pjo_ref_slot.argtypes = I32, [U32, I32]
        L.pjo_digits.restype = None
        L.pjo_digits.argtypes = [P, I64, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, P]
        L.pjo_histogram.restype = None
        L.pjo_histogram.argtypes = [P, I64, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, P]
        L.pjo_inner_join.restype = I64
        L.pjo_inner_join.argtypes = [P, I64, P, I64, ctypes.c_int, ctypes.c_int, P, P, I64]
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _keys(a) -> np.ndarray:
    a = np.ascontiguousarray(a)
    if a.dtype not in (np.int32, np.int64):
        raise TypeError("keys must be int32 or int64")
    return a


def hash_keys(keys) -> np.ndarray:
    """MurmurHash3_x86_32 (seed 0) of every key: hash_functions.cuh:80-119."""
    k = _keys(keys)
    out = np.empty(k.shape[0], dtype=np.uint32)
    lib().pjo_hash_array(_ptr(k), k.shape[0], k.itemsize, _ptr(out))
    return out


def ref_slot(h: int, table_size: int) -> int:
    """abs((int)h % T): hash_join_kernels.cuh:100-101."""
    return lib().pjo_ref_slot(h, table_size)


DIGIT_RAW, DIGIT_HASH = 0, 1


def digits(keys, mode: int, b1: int, b2: int = 0, which: int = 0) -> np.ndarray:
    """Partition digit of every key (partition_kernels.cuh:168,380 for mode 0)."""
    k = _keys(keys)
    out = np.empty(k.shape[0], dtype=np.int32)
    lib().pjo_digits(_ptr(k), k.shape[0], k.itemsize, mode, b1, b2, which, _ptr(out))
    return out


def histogram(keys, mode: int, b1: int, b2: int = 0, which: int = 0) -> np.ndarray:
    k = _keys(keys)
    nb = b1 if which == 1 else b2 if which == 2 else b1 + b2
    out = np.empty(1 << nb, dtype=np.int32)
    lib().pjo_histogram(_ptr(k), k.shape[0], k.itemsize, mode, b1, b2, which, _ptr(out))
    return out


def inner_join(build_keys, probe_keys, unique_keys: bool = True):
    """(build_row, probe_row) pairs of inner_join_cpu (inner_join_cpu.hpp:24-107)."""
    b, p = _keys(build_keys), _keys(probe_keys)
    if b.dtype != p.dtype:
        raise TypeError("build and probe keys must have the same dtype")
    L = lib()
    total = L.pjo_inner_join(_ptr(b), b.shape[0], _ptr(p), p.shape[0], b.itemsize, int(unique_keys),
                             None, None, 0)
    if total < 0:
        raise MemoryError("oracle join: allocation failed")
    br = np.empty(total, dtype=np.int32)
    pr = np.empty(total, dtype=np.int32)
    got = L.pjo_inner_join(_ptr(b), b.shape[0], _ptr(p), p.shape[0], b.itemsize, int(unique_keys),
                           _ptr(br), _ptr(pr), total)
    assert got == total
    return br, pr


def sorted_pairs(build_row, probe_row) -> np.ndarray:
    """Pairs as one int64 per pair, sorted: the multiset comparison of
    check_results (inner_join_cpu.hpp:110-168) without its key projection."""
    b = np.asarray(build_row, dtype=np.int64)
    p = np.asarray(probe_row, dtype=np.int64)
    return np.sort((b << 32) | (p & 0xFFFFFFFF))


# ---------------------------------------------------------------------------
# The reference's own code, compiled by oracle/build_ref.sh into oracle/_ref.

_ref_cpu = None


def ref_cpu_available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "libref_cpu.so"))


def ref_cpu():
    global _ref_cpu
    if _ref_cpu is None:
        L = ctypes.CDLL(os.path.join(REF_DIR, "libref_cpu.so"))
        P, I64, I32, U32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_uint32
        L.ref_murmur_i32.restype, L.ref_murmur_i32.argtypes = U32, [I32]
        L.ref_murmur_i64.restype, L.ref_murmur_i64.argtypes = U32, [I64]
        L.ref_slot.restype, L.ref_slot.argtypes = I32, [U32, I32]
        for name in ("ref_inner_join_cpu_i32", "ref_inner_join_cpu_i64"):
            f = getattr(L, name)
            f.restype = I64
            f.argtypes = [P, I64, P, I64, ctypes.c_int, P, I64, ctypes.POINTER(ctypes.c_double), ctypes.c_int]
        L.ref_omp_max_threads.restype = ctypes.c_int
        _ref_cpu = L
    return _ref_cpu


def ref_inner_join_cpu(build_keys, probe_keys, unique_keys: bool = True, threads: int = 0):
    """Run the reference's inner_join_cpu; returns (keys of the emitted
    records, seconds measured by the function itself)."""
    b, p = _keys(build_keys), _keys(probe_keys)
    L = ref_cpu()
    f = L.ref_inner_join_cpu_i32 if b.dtype == np.int32 else L.ref_inner_join_cpu_i64
    sec = ctypes.c_double(0.0)
    cap = p.shape[0] if unique_keys else 0
    out = np.empty(max(cap, 1), dtype=b.dtype)
    n = f(_ptr(b), b.shape[0], _ptr(p), p.shape[0], int(unique_keys), _ptr(out), cap, ctypes.byref(sec), threads)
    if n > cap:
        out = np.empty(n, dtype=b.dtype)
        n = f(_ptr(b), b.shape[0], _ptr(p), p.shape[0], int(unique_keys), _ptr(out), n, ctypes.byref(sec), threads)
    return out[:n], sec.value


_ref_gpu = {}


def ref_gpu_available(key_bytes: int = 4) -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"libref_gpu_k{key_bytes}.so"))


def ref_gpu(key_bytes: int = 4):
    if key_bytes not in _ref_gpu:
        L = ctypes.CDLL(os.path.join(REF_DIR, f"libref_gpu_k{key_bytes}.so"))
        P, I = ctypes.c_void_p, ctypes.c_int
        L.ref_gpu_partitioned_join.restype = I
        L.ref_gpu_partitioned_join.argtypes = [P, I, P, I, P, P, I, I, I, I, ctypes.c_float, I, I, P, P, P, P]
        L.ref_gpu_key_bytes.restype = I
        _ref_gpu[key_bytes] = L
    return _ref_gpu[key_bytes]


def ref_gpu_partitioned_join(build_keys, probe_keys, probe_rows_as_values=True, unique_keys=True,
                             radix=True, p1=256, p2=512, factor=1.0, combined_histo=False,
                             capacity=None):
    """Drive the reference's GPU stages (main.cu:762-892) on these inputs.

    With probe_rows_as_values the probe payload column is the probe row id
    and the build payload the build row id (-V), so the records' .y field is
    the probe row.  Returns (keys, y, stage_ms[6])."""
    b, p = _keys(build_keys), _keys(probe_keys)
    L = ref_gpu(b.itemsize)
    if capacity is None:
        capacity = max(1, int(lib().pjo_inner_join(_ptr(b), b.shape[0], _ptr(p), p.shape[0], b.itemsize,
                                                   int(unique_keys), None, None, 0)))
    vb = vp = None
    if probe_rows_as_values:
        vb = np.arange(b.shape[0], dtype=b.dtype)
        vp = np.arange(p.shape[0], dtype=b.dtype)
    out_x = np.empty(capacity, dtype=b.dtype)
    out_y = np.empty(capacity, dtype=b.dtype)
    cnt = np.zeros(1, dtype=np.int32)
    ms = np.zeros(6, dtype=np.float32)
    rc = L.ref_gpu_partitioned_join(_ptr(b), b.shape[0], _ptr(p), p.shape[0],
                                    None if vb is None else _ptr(vb), None if vp is None else _ptr(vp),
                                    int(unique_keys), int(radix), p1, p2, float(factor), int(combined_histo),
                                    capacity, _ptr(out_x), _ptr(out_y), _ptr(cnt), _ptr(ms))
    if rc != 0:
        raise RuntimeError(f"reference GPU path refused or failed: code {rc}")
    n = min(int(cnt[0]), capacity)
    return out_x[:n], out_y[:n], ms
