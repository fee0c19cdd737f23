"""Generates tests/golden/golden_ref.npz from the reference's own code.

Run in a container that has the reference tree: it needs
oracle/_ref/libref_cpu.so, which oracle/build_ref.sh compiles from the
reference's src/hash_functions.cuh, src/int_fastdiv.h and
src/inner_join_cpu.hpp.  The fixture it writes is committed; the tests read
it on any machine (the reference tree is not needed at test time).

Contents (all produced by the reference's code, never by the oracle):
  hash_i32_keys / hash_i32      MurmurHash3_32<int>        (hash_functions.cuh:80-119)
  hash_i64_keys / hash_i64      MurmurHash3_32<long long>
  slot_h / slot_T / slot        abs((int)h % T) through int_fastdiv (hash_join_kernels.cuh:100-101)
  join_<case>_build / _probe    seeded inputs
  join_<case>_keys              sorted keys of inner_join_cpu's records (inner_join_cpu.hpp:24-107)
  join_<case>_unique            the uniq_keys flag used
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden_ref.npz")


def edge_i32():
    return np.array([0, 1, -1, 2, 42, 0x7FFFFFFF, -0x80000000, 0x7FFFFFFE, -2, 1 << 20, 1 << 27,
                     (1 << 27) + 1, 0x55555555, -0x55555556], dtype=np.int32)


def edge_i64():
    return np.array([0, 1, -1, 42, (1 << 63) - 1, -(1 << 63), 1 << 32, (1 << 32) - 1, -(1 << 32),
                     0x0123456789ABCDEF, -0x0123456789ABCDEF, 1 << 40, 123456789012345], dtype=np.int64)


def join_cases(rng):
    cases = {}
    # int32, unique build keys (a permutation), 70 % of probes match.
    b = (rng.permutation(3000) + 1).astype(np.int32)
    miss = rng.integers(10_000, 20_000, size=7000).astype(np.int32)
    hit = b[rng.integers(0, b.shape[0], size=7000)]
    p = np.where(rng.random(7000) < 0.7, hit, miss).astype(np.int32)
    cases["i32_unique"] = (b, p, True)
    # int32, repeated build keys, multimap semantics.
    b = rng.integers(0, 700, size=2500).astype(np.int32)
    p = rng.integers(0, 1000, size=3000).astype(np.int32)
    cases["i32_multi"] = (b, p, False)
    # int32, repeated build keys under the unique flag (map keeps the first row).
    cases["i32_unique_flag_dups"] = (b, p, True)
    # int32 extremes, sentinel-looking keys included (-1 is joinable on the CPU).
    e = edge_i32()
    b = np.concatenate([e, (rng.permutation(500) + 100).astype(np.int32)])
    p = np.concatenate([e, e[::-1], rng.integers(0, 800, size=900).astype(np.int32)])
    cases["i32_edges"] = (b, p, True)
    # int64 unique random keys, skewed probes with misses.
    b = np.unique(rng.integers(-(1 << 62), 1 << 62, size=4000, dtype=np.int64))
    b = b[rng.permutation(b.shape[0])]
    ranks = np.minimum(rng.zipf(1.3, size=8000) - 1, b.shape[0] - 1)
    p = b[ranks].copy()
    m = rng.random(8000) < 0.2
    p[m] = rng.integers(-(1 << 62), 1 << 62, size=int(m.sum()), dtype=np.int64)
    cases["i64_unique_zipf"] = (b, p, True)
    # int64 multimap with extremes.
    e = edge_i64()
    b = np.concatenate([e, e[:5], rng.integers(0, 300, size=1500).astype(np.int64)])
    p = np.concatenate([e, rng.integers(0, 400, size=2000).astype(np.int64)])
    cases["i64_multi"] = (b, p, False)
    # no match at all, and a one-row build side.
    cases["i32_nomatch"] = (np.arange(1, 1001, dtype=np.int32), np.arange(2001, 3001, dtype=np.int32), True)
    cases["i32_single"] = (np.array([7], dtype=np.int32), np.array([7, 8, 7, 7, 0], dtype=np.int32), True)
    return cases


def main():
    if not oracle.ref_cpu_available():
        raise SystemExit("oracle/_ref/libref_cpu.so missing: run oracle/build_ref.sh where the reference tree exists")
    R = oracle.ref_cpu()
    rng = np.random.default_rng(20240611)
    out = {}

    k32 = np.concatenate([edge_i32(), rng.integers(-(1 << 31), 1 << 31, size=4096).astype(np.int32)])
    out["hash_i32_keys"] = k32
    out["hash_i32"] = np.array([R.ref_murmur_i32(int(k)) for k in k32], dtype=np.uint32)
    k64 = np.concatenate([edge_i64(), rng.integers(-(1 << 63), (1 << 63) - 1, size=4096, dtype=np.int64)])
    out["hash_i64_keys"] = k64
    out["hash_i64"] = np.array([R.ref_murmur_i64(int(k)) for k in k64], dtype=np.uint32)

    h = np.concatenate([np.array([0, 1, 0x7FFFFFFF, 0x80000000, 0xFFFFFFFF], dtype=np.uint64),
                        rng.integers(0, 1 << 32, size=4096, dtype=np.uint64)]).astype(np.uint32)
    T = np.concatenate([np.array([1, 2, 3, 0x7FFFFFFF, 7], dtype=np.int64),
                        np.where(rng.random(4096) < 0.5, rng.integers(1, 1 << 16, size=4096),
                                 rng.integers(1, (1 << 31) - 1, size=4096))]).astype(np.int32)
    out["slot_h"], out["slot_T"] = h, T
    out["slot"] = np.array([R.ref_slot(int(a), int(b)) for a, b in zip(h, T)], dtype=np.int32)

    for name, (b, p, uniq) in join_cases(rng).items():
        keys, _ = oracle.ref_inner_join_cpu(b, p, uniq, threads=4)
        out[f"join_{name}_build"] = b
        out[f"join_{name}_probe"] = p
        out[f"join_{name}_keys"] = np.sort(keys)
        out[f"join_{name}_unique"] = np.array(uniq)
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT}: {len(out)} arrays, {os.path.getsize(OUT)} bytes")


if __name__ == "__main__":
    main()
