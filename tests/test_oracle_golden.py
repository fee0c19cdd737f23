"""Pins the oracle against golden vectors made by the reference's own code
(tests/golden/make_golden.py over oracle/_ref/libref_cpu.so)."""
import numpy as np
import pytest

from oracle import oracle

JOIN_CASES = ["i32_unique", "i32_multi", "i32_unique_flag_dups", "i32_edges", "i64_unique_zipf",
              "i64_multi", "i32_nomatch", "i32_single"]


def test_hash_i32_matches_reference(golden):
    assert np.array_equal(oracle.hash_keys(golden["hash_i32_keys"]), golden["hash_i32"])


def test_hash_i64_matches_reference(golden):
    assert np.array_equal(oracle.hash_keys(golden["hash_i64_keys"]), golden["hash_i64"])


def test_known_hash_values():
    # MurmurHash3_x86_32 seed 0 of the 4-byte keys 0, 1, 42 (recomputed by
    # the reference header in make_golden.py; repeated here as literals).
    assert [int(x) for x in oracle.hash_keys(np.array([0, 1, 42], np.int32))] == [0x2362F9DE, 0xFBF1402A, 0xBC5B91E3]


def test_ref_slot_matches_reference(golden):
    got = np.array([oracle.ref_slot(int(h), int(t)) for h, t in zip(golden["slot_h"], golden["slot_T"])])
    assert np.array_equal(got, golden["slot"])


@pytest.mark.parametrize("case", JOIN_CASES)
def test_inner_join_matches_reference(golden, case):
    b = golden[f"join_{case}_build"]
    p = golden[f"join_{case}_probe"]
    uniq = bool(golden[f"join_{case}_unique"])
    br, pr = oracle.inner_join(b, p, uniq)
    # every pair is a real match
    assert np.array_equal(b[br], p[pr])
    # key projection equals the reference's {key, 0} record multiset
    assert np.array_equal(np.sort(b[br]), golden[f"join_{case}_keys"])
    # each probe row appears at most once under the unique flag
    if uniq:
        assert np.unique(pr).shape[0] == pr.shape[0]


def test_histogram_raw_digits_follow_reference_formula():
    rng = np.random.default_rng(3)
    k = rng.integers(-(1 << 31), 1 << 31, size=20000).astype(np.int32)
    b1, b2 = 5, 3
    d1 = oracle.digits(k, oracle.DIGIT_RAW, b1, b2, which=1)
    d2 = oracle.digits(k, oracle.DIGIT_RAW, b1, b2, which=2)
    # partition_kernels.cuh:168 and :380 evaluated in numpy
    exp1 = ((((1 << b1) - 1) << b2) & k.astype(np.int64)) >> b2
    exp2 = k.astype(np.int64) & ((1 << b2) - 1)
    assert np.array_equal(d1, exp1) and np.array_equal(d2, exp2)
    h = oracle.histogram(k, oracle.DIGIT_RAW, b1, b2, which=0)
    assert h.sum() == k.shape[0]
    assert np.array_equal(h, np.bincount((exp1 << b2) | exp2, minlength=1 << (b1 + b2)))


def test_histogram_hash_digits_are_top_bits():
    rng = np.random.default_rng(4)
    k = rng.integers(-(1 << 62), 1 << 62, size=5000, dtype=np.int64)
    h = oracle.hash_keys(k).astype(np.int64)
    assert np.array_equal(oracle.digits(k, oracle.DIGIT_HASH, 7, 4, which=0), h >> 21)
    assert np.array_equal(oracle.digits(k, oracle.DIGIT_HASH, 7, 4, which=1), h >> 25)
    assert np.array_equal(oracle.digits(k, oracle.DIGIT_HASH, 7, 4, which=2), (h >> 21) & 15)
