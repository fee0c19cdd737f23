"""Parity of the CUDA path (through the C ABI) with the oracle and with the
reference's golden vectors.  Bit-exact: integer and index work."""
import numpy as np
import pytest
import torch

from oracle import oracle
from partitioned_join_b200 import (DIGIT_HASH, DIGIT_RAW, SLOT_FAST, SLOT_REF, SPLIT_HASH, SPLIT_POSITION, TABLE_BUCKET,
                                   TABLE_COMPACT, TABLE_EXACT, TABLE_OPEN, PJError)
from partitioned_join_b200 import api, datagen

pytestmark = pytest.mark.gpu

DEV = "cuda:0"


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def pairs_equal(b, p, br, pr, unique=True):
    """Sorted multiset of (build_row, probe_row) equals the oracle's."""
    eb, ep = oracle.inner_join(b, p, unique)
    got = oracle.sorted_pairs(br.cpu().numpy(), pr.cpu().numpy())
    exp = oracle.sorted_pairs(eb, ep)
    return got.shape == exp.shape and np.array_equal(got, exp)


def run(b, p, unique=True, plan=None):
    br, pr = api.partitioned_join(dev(b), dev(p), unique_build_keys=unique, plan=plan)
    torch.cuda.synchronize()
    return br, pr


# ---------------------------------------------------------------------------
# hash, slot and digit functions against the reference's golden vectors

def test_hash_matches_reference_golden(golden):
    for kind in ("i32", "i64"):
        keys = golden[f"hash_{kind}_keys"]
        got = api.hash_keys(dev(keys)).cpu().numpy().view(np.uint32)
        assert np.array_equal(got, golden[f"hash_{kind}"]), kind


def test_ref_slot_matches_oracle():
    rng = np.random.default_rng(5)
    keys = rng.integers(-(1 << 31), 1 << 31, size=20000).astype(np.int32)
    h = oracle.hash_keys(keys)
    for T in (1, 7, 1000, 12289, 16384, 2**31 - 1):
        got = api.hash_slots(dev(keys), T, SLOT_REF).cpu().numpy()
        exp = np.array([oracle.ref_slot(int(x), T) for x in h[:2000]])
        assert np.array_equal(got[:2000], exp), T
        assert got.min() >= 0 and got.max() < T


def test_fast_slot_in_range():
    rng = np.random.default_rng(6)
    keys = rng.integers(-(1 << 62), 1 << 62, size=50000, dtype=np.int64)
    for T, skip in ((1000, 0), (16384, 12), (8191, 20)):
        got = api.hash_slots(dev(keys), T, SLOT_FAST, skip).cpu().numpy()
        h = oracle.hash_keys(keys).astype(np.uint64)
        exp = (((h << np.uint64(skip)) & np.uint64(0xFFFFFFFF)) * np.uint64(T)) >> np.uint64(32)
        assert np.array_equal(got.astype(np.uint64), exp)


@pytest.mark.parametrize("mode", [DIGIT_RAW, DIGIT_HASH])
@pytest.mark.parametrize("dtype", [np.int32, np.int64])
def test_radix_histogram_matches_oracle(mode, dtype):
    rng = np.random.default_rng(7)
    info = np.iinfo(dtype)
    keys = rng.integers(info.min, info.max, size=300001, dtype=dtype)
    for b1, b2, which in ((0, 0, 0), (1, 0, 0), (10, 0, 0), (5, 3, 1), (5, 3, 2), (6, 6, 0), (14, 0, 0)):
        got = api.radix_histogram(dev(keys), mode, b1, b2, which).cpu().numpy()
        exp = oracle.histogram(keys, mode, b1, b2, which)
        assert np.array_equal(got, exp), (b1, b2, which)


# ---------------------------------------------------------------------------
# the partition stage: every partition holds exactly the rows whose digit it is

@pytest.mark.parametrize("dtype", [np.int32, np.int64])
@pytest.mark.parametrize("bits", [0, 3, 9])
@pytest.mark.parametrize("mode", [DIGIT_RAW, DIGIT_HASH])
def test_partition_stage_exact(dtype, bits, mode):
    rng = np.random.default_rng(8 + bits)
    n = 200003
    info = np.iinfo(dtype)
    keys = rng.integers(info.min // 2, info.max // 2, size=n, dtype=dtype)
    plan = api.plan_default(n, n, np.dtype(dtype).itemsize)
    plan.bits1 = bits
    plan.wc_tuples = 4 if dtype == np.int32 else 2   # the default's width may not fit 2^9 buffers
    plan.digit_mode = mode
    tuples, offsets = api.partition(dev(keys), plan)
    t = tuples.cpu().numpy()
    off = offsets.cpu().numpy()
    words = 2 if dtype == np.int32 else 4
    P = 1 << bits
    assert off[0] == 0 and np.all(np.diff(off) >= 0)
    rec = t[: off[-1] * words].reshape(-1, words)
    rows = rec[:, -1]
    real = rows >= 0
    if dtype == np.int32:
        # 4-byte keys are stored as murmur(key), a bijection of 32-bit values
        k = rec[:, 0].astype(np.uint32)
        assert np.array_equal(k[real], oracle.hash_keys(keys[rows[real]]))
    else:
        k = (rec[:, 1].astype(np.int64) << 32) | (rec[:, 0].astype(np.int64) & 0xFFFFFFFF)
        assert np.array_equal(k[real], keys[rows[real]])
        assert np.array_equal(rec[real, 2].astype(np.uint32), oracle.hash_keys(keys[rows[real]]))
    assert np.all(rows[~real] == -1)
    # every input row exactly once
    assert np.array_equal(np.sort(rows[real]), np.arange(n))
    # every row sits in its digit's partition
    part = np.repeat(np.arange(P), np.diff(off))
    d = oracle.digits(keys, mode, bits, 0, 0)
    assert np.array_equal(part[real], d[rows[real]])


@pytest.mark.parametrize("dtype", [np.int32, np.int64])
@pytest.mark.parametrize("mode", [DIGIT_RAW, DIGIT_HASH])
def test_two_pass_partition_stage_exact(dtype, mode):
    rng = np.random.default_rng(31)
    n = 300007
    info = np.iinfo(dtype)
    keys = rng.integers(info.min // 2, info.max // 2, size=n, dtype=dtype)
    plan = api.plan_default(n, n, np.dtype(dtype).itemsize)
    plan.passes, plan.bits1, plan.bits2, plan.digit_mode = 2, 3, 4, mode
    tuples, offsets = api.partition(dev(keys), plan)
    t, off = tuples.cpu().numpy(), offsets.cpu().numpy()
    words = 2 if dtype == np.int32 else 4
    P1, P2 = 8, 16
    assert off.shape[0] == P1 * P2 + 1 and off[0] == 0 and np.all(np.diff(off) >= 0)
    rec = t[: off[-1] * words].reshape(-1, words)
    rows = rec[:, -1]
    real = rows >= 0
    assert np.array_equal(np.sort(rows[real]), np.arange(n))
    # partition q = p2 * P1 + p1: p1 the first-pass digit, p2 the next hash bits
    q = np.repeat(np.arange(P1 * P2), np.diff(off))
    h = oracle.hash_keys(keys).astype(np.int64)
    p1 = oracle.digits(keys, mode, 3, 0, 0).astype(np.int64)
    hb = 3 if mode == DIGIT_HASH else 0
    p2 = (h >> (32 - hb - 4)) & (P2 - 1)
    assert np.array_equal(q[real], (p2 * P1 + p1)[rows[real]])


@pytest.mark.parametrize("dtype", [np.int32, np.int64])
@pytest.mark.parametrize("mode", [DIGIT_RAW, DIGIT_HASH])
@pytest.mark.parametrize("unique", [True, False])
def test_two_pass_join_matches_oracle(dtype, mode, unique):
    b, p = datagen.config2(seed=32, n_build=400000, n_probe=700000)
    b, p = b.astype(dtype), p.astype(dtype)
    if not unique:
        b = np.concatenate([b, b[:30000]])
    plan = api.plan_default(b.shape[0], p.shape[0], np.dtype(dtype).itemsize, unique)
    plan.passes, plan.bits1, plan.bits2, plan.digit_mode = 2, 3, 4, mode
    plan.table_mode, plan.table_capacity = TABLE_BUCKET, 8192
    br, pr = run(b, p, unique, plan)
    assert pairs_equal(b, p, br, pr, unique)


def test_two_pass_default_plan_for_large_builds():
    plan = api.plan_default(1 << 29, 1 << 29, 4)
    assert plan.passes == 2 and plan.bits1 + plan.bits2 >= 14 and plan.table_mode == TABLE_BUCKET


# ---------------------------------------------------------------------------
# full join parity against the oracle

@pytest.mark.parametrize("case", ["i32_unique", "i32_multi", "i32_unique_flag_dups", "i32_edges",
                                  "i64_unique_zipf", "i64_multi", "i32_nomatch", "i32_single"])
def test_join_golden_cases(golden, case):
    b = golden[f"join_{case}_build"]
    p = golden[f"join_{case}_probe"]
    uniq = bool(golden[f"join_{case}_unique"])
    br, pr = run(b, p, uniq)
    bk = b[br.cpu().numpy()]
    # key projection equals the reference inner_join_cpu's record multiset
    assert np.array_equal(np.sort(bk), golden[f"join_{case}_keys"])
    if case != "i32_unique_flag_dups":
        assert pairs_equal(b, p, br, pr, uniq)
    else:
        # repeated keys under the unique flag: each probe row matches one of them
        assert np.array_equal(b[br.cpu().numpy()], p[pr.cpu().numpy()])


def test_join_config1_shape_scaled():
    b, p = datagen.config1(seed=11, n_build=1 << 18, n_probe=1 << 20)
    br, pr = run(b, p)
    assert br.numel() == p.shape[0]
    assert pairs_equal(b, p, br, pr)


def test_join_config2_shape_scaled():
    b, p = datagen.config2(seed=12, n_build=1 << 21, n_probe=1 << 21)
    br, pr = run(b, p)
    assert pairs_equal(b, p, br, pr)


@pytest.mark.parametrize("digit", [DIGIT_RAW, DIGIT_HASH])
@pytest.mark.parametrize("table,slot", [(TABLE_BUCKET, SLOT_FAST), (TABLE_COMPACT, SLOT_FAST), (TABLE_OPEN, SLOT_FAST),
                                        (TABLE_OPEN, SLOT_REF)])
@pytest.mark.parametrize("split", [SPLIT_HASH, SPLIT_POSITION])
@pytest.mark.parametrize("dtype", [np.int32, np.int64])
def test_join_plan_variants(digit, table, slot, split, dtype):
    b, p = datagen.config2(seed=13, n_build=300000, n_probe=500000)
    b, p = b.astype(dtype), p.astype(dtype)
    if dtype == np.int64:
        b = b * 7919 - (1 << 40)
        p = p * 7919 - (1 << 40)
    plan = api.plan_default(b.shape[0], p.shape[0], np.dtype(dtype).itemsize)
    plan.digit_mode, plan.table_mode, plan.slot_mode, plan.split_mode = digit, table, slot, split
    plan.bits1 = 3                  # coarse: forces several pieces per partition
    plan.table_capacity = 8192
    plan.probe_chunk = 4096         # several probe chunks per partition
    br, pr = run(b, p, True, plan)
    assert pairs_equal(b, p, br, pr)


def _fingerprint_twins(dtype, n_pairs, bits=23):
    """Pairs of distinct keys whose hashes agree on the low `bits` bits."""
    keys = (np.arange(1, 1 << 22, dtype=np.int64) * 2654435761 + 12345).astype(dtype)
    low = oracle.hash_keys(keys).astype(np.int64) & ((1 << bits) - 1)
    order = np.argsort(low, kind="stable")
    ls = low[order]
    same = np.nonzero(ls[1:] == ls[:-1])[0]
    a, b = keys[order[same]], keys[order[same + 1]]
    # one pair per low value, pairs disjoint
    _, first = np.unique(ls[same], return_index=True)
    a, b = a[first], b[first]
    used = set()
    pa, pb = [], []
    for x, y in zip(a.tolist(), b.tolist()):
        if x in used or y in used:
            continue
        used.update((x, y))
        pa.append(x)
        pb.append(y)
        if len(pa) == n_pairs:
            break
    return np.array(pa, dtype=dtype), np.array(pb, dtype=dtype)


@pytest.mark.parametrize("dtype", [np.int32, np.int64])
@pytest.mark.parametrize("unique", [True, False])
def test_join_compact_fingerprint_collisions(dtype, unique):
    # a 2^7-bucket COMPACT table compares 7 bucket + 16 fingerprint hash
    # bits: probe keys built to agree with a build key on those 23 bits but
    # not on the key must be rejected by the full-key check, and the walk
    # must go on to the true match when there is one
    a, b = _fingerprint_twins(dtype, 3000)
    build = np.concatenate([a, b[:1000]])           # some twins are both present
    if not unique:
        build = np.concatenate([build, a[:500]])
    probe = np.concatenate([b, a, b[:1000]])
    rng = np.random.default_rng(23)
    rng.shuffle(build)
    rng.shuffle(probe)
    plan = api.plan_default(build.shape[0], probe.shape[0], np.dtype(dtype).itemsize, unique)
    plan.table_mode, plan.digit_mode, plan.bits1 = TABLE_COMPACT, DIGIT_RAW, 0
    plan.split_mode = SPLIT_POSITION
    plan.table_capacity = 256                      # 2^7 buckets
    br, pr = run(build, probe, unique, plan)
    assert pairs_equal(build, probe, br, pr, unique)


@pytest.mark.parametrize("dtype", [np.int32, np.int64])
@pytest.mark.parametrize("unique", [True, False])
@pytest.mark.parametrize("split", [SPLIT_HASH, SPLIT_POSITION])
@pytest.mark.parametrize("n_build", [4096, 4097, 300007])
def test_join_exact_tables_match_oracle(dtype, unique, split, n_build):
    # EXACT entries hold the build row in the low bits (12, 13 and 19 row
    # bits here) and the hash bits above the bucket bits (8-byte keys: and
    # the key's low word); small tables force several pieces per partition
    rng = np.random.default_rng(n_build)
    b = rng.permutation(np.arange(1, 3 * n_build, 3, dtype=np.int64))[:n_build]
    if dtype == np.int64:
        b = b * 0x100000001 + (b % 7) * (1 << 40)   # high words matter
    b = b.astype(dtype)
    if not unique:
        b[: n_build // 10] = b[n_build // 10: 2 * (n_build // 10)]
    info = np.iinfo(dtype)
    p = np.concatenate([rng.choice(b, 2 * n_build), rng.integers(info.min, info.max, n_build)]).astype(dtype)
    plan = api.plan_default(n_build, p.shape[0], np.dtype(dtype).itemsize, unique)
    plan.table_mode, plan.digit_mode, plan.split_mode = TABLE_EXACT, DIGIT_HASH, split
    plan.bits1 = 4
    plan.wc_tuples = 4
    plan.table_capacity = 2048
    plan.probe_chunk = 4096
    br, pr = run(b, p, unique, plan)
    assert pairs_equal(b, p, br, pr, unique)


@pytest.mark.parametrize("mode", [DIGIT_RAW, DIGIT_HASH])
def test_join_exact_tables_two_pass(mode):
    # the join partition of a two-pass plan fixes bits2 hash bits (and the
    # bits1 above them with hash digits): EXACT entries count on them
    b, p = datagen.config2(seed=36, n_build=400000, n_probe=700000)
    plan = api.plan_default(b.shape[0], p.shape[0], 4)
    plan.passes, plan.bits1, plan.bits2, plan.digit_mode = 2, 4, 6, mode
    plan.table_mode, plan.table_capacity = TABLE_EXACT, 4096
    br, pr = run(b, p, True, plan)
    assert pairs_equal(b, p, br, pr)


def test_join_exact_tables_with_heavy_keys():
    rng = np.random.default_rng(37)
    b = rng.permutation(400000).astype(np.int32)
    p = np.concatenate([rng.integers(0, 500000, size=600000), np.full(200000, 17), np.full(50000, 450001)]).astype(np.int32)
    rng.shuffle(p)
    plan = api.plan_default(b.shape[0], p.shape[0], 4)
    plan.table_mode, plan.digit_mode, plan.bits1, plan.wc_tuples = TABLE_EXACT, DIGIT_HASH, 5, 4
    plan.table_capacity = 16384
    plan.set_heavy([17, 450001])
    br, pr = run(b, p, True, plan)
    assert pairs_equal(b, p, br, pr)


def test_join_exact_tables_hash_twins():
    # keys whose hashes agree on all bits below the partition digits: the
    # digits alone tell them apart, and EXACT entries must not confuse them
    keys = (np.arange(1, 1 << 22, dtype=np.int64) * 2654435761 + 12345).astype(np.int32)
    h = oracle.hash_keys(keys).astype(np.int64)
    low = h & ((1 << 26) - 1)
    order = np.argsort(low, kind="stable")
    ls = low[order]
    same = np.nonzero(ls[1:] == ls[:-1])[0]
    a, c = keys[order[same]], keys[order[same + 1]]
    keep = np.unique(np.concatenate([a, c]), return_index=True)[1]
    twins = np.concatenate([a, c])[np.sort(keep)]
    assert len(twins) > 100
    build = twins[::2]
    probe = np.concatenate([twins, keys[:5000]])
    build = np.unique(build)
    plan = api.plan_default(build.shape[0], probe.shape[0], 4)
    plan.table_mode, plan.digit_mode, plan.bits1, plan.wc_tuples = TABLE_EXACT, DIGIT_HASH, 6, 4
    plan.table_capacity = 1024
    br, pr = run(build, probe, True, plan)
    assert pairs_equal(build, probe, br, pr)


def test_join_exact_tables_int64_same_low_words():
    # 8-byte keys that share their low word and differ only in the high
    # word: the entry's low word and hash bits still tell them apart
    lo = np.arange(1, 2001, dtype=np.int64)
    keys = np.concatenate([lo + (h << 32) for h in range(1, 41)])      # 40 keys per low word
    rng = np.random.default_rng(38)
    rng.shuffle(keys)
    build = keys[::2]
    probe = np.concatenate([keys, keys[:5000]])
    plan = api.plan_default(build.shape[0], probe.shape[0], 8)
    plan.table_mode, plan.digit_mode, plan.bits1, plan.wc_tuples = TABLE_EXACT, DIGIT_HASH, 3, 2
    plan.table_capacity = 4096
    br, pr = run(build, probe, True, plan)
    assert pairs_equal(build, probe, br, pr)


def test_join_exact_tables_planned_where_they_fit():
    assert api.plan_default(1 << 27, 1 << 27, 4).table_mode == TABLE_EXACT
    assert api.plan_default(1 << 26, 1 << 28, 8).table_mode == TABLE_EXACT
    # 32 K-tuple partitions of 8-byte keys exceed an EXACT table's ~22 K
    assert api.plan_default(1 << 27, 1 << 27, 8).table_mode == TABLE_COMPACT


def test_join_exact_tables_rejected_where_inexact():
    b32 = np.arange(1, 1 << 20, dtype=np.int32)
    plan = api.plan_default(b32.shape[0], b32.shape[0], 4)
    plan.table_mode, plan.digit_mode, plan.bits1, plan.wc_tuples = TABLE_EXACT, DIGIT_RAW, 0, 4
    plan.table_capacity = 1024
    with pytest.raises(PJError):             # 2^20 buckets needed: no room
        run(b32, b32, True, plan)


def test_join_compact_default_plan_large_partitions():
    # past one pass's fan-out the default plan takes COMPACT tables
    b, p = datagen.config2(seed=22, n_build=1 << 22, n_probe=1 << 22)
    plan = api.plan_default(b.shape[0], p.shape[0], 4)
    plan.table_mode = TABLE_COMPACT
    plan.table_capacity = 41472 // 128 * 128
    plan.bits1 = 7                 # 32 K build tuples per partition, no split
    br, pr = run(b, p, True, plan)
    assert pairs_equal(b, p, br, pr)


@pytest.mark.parametrize("w", [2, 4, 8, 16, 32])
def test_join_wc_widths(w):
    b, p = datagen.config2(seed=18, n_build=200000, n_probe=300000)
    plan = api.plan_default(b.shape[0], p.shape[0], 4)
    plan.wc_tuples = w
    plan.bits1 = 7
    br, pr = run(b, p, True, plan)
    assert pairs_equal(b, p, br, pr)


def test_join_int64_skewed():
    b, p = datagen.config3(seed=14, theta=1.25, n_build=1 << 17, n_probe=1 << 19)
    br, pr = run(b, p)
    assert pairs_equal(b, p, br, pr)


def test_join_multimap_heavy_duplicates():
    rng = np.random.default_rng(15)
    b = np.concatenate([np.full(5000, 77, np.int32), rng.integers(0, 20000, size=30000).astype(np.int32)])
    p = np.concatenate([np.full(300, 77, np.int32), rng.integers(0, 30000, size=60000).astype(np.int32)])
    br, pr = run(b, p, unique=False)
    assert pairs_equal(b, p, br, pr, unique=False)


def test_join_all_probes_one_key():
    b = np.arange(1, 100001, dtype=np.int32)
    p = np.full(400000, 4242, dtype=np.int32)
    br, pr = run(b, p)
    assert pairs_equal(b, p, br, pr)


def test_join_sentinel_keys_join():
    # -1 is the reference's empty-slot marker; here it is an ordinary key
    b = np.array([-1, 0, 1, -2**31, 2**31 - 1], dtype=np.int32)
    p = np.array([-1, -1, 2**31 - 1, 5, 0, -2**31], dtype=np.int32)
    br, pr = run(b, p)
    assert pairs_equal(b, p, br, pr)


def test_join_empty_sides():
    e = np.zeros(0, np.int32)
    x = np.arange(100, dtype=np.int32)
    for b, p in ((e, x), (x, e), (e, e)):
        br, pr = run(b, p)
        assert br.numel() == 0 and pr.numel() == 0


def test_join_ragged_sizes():
    rng = np.random.default_rng(16)
    for nb, np_ in ((1, 1), (3, 17), (15, 33), (1023, 4097), (70001, 130003)):
        b = rng.permutation(nb * 3)[:nb].astype(np.int32)
        p = rng.integers(0, nb * 3, size=np_).astype(np.int32)
        br, pr = run(b, p)
        assert pairs_equal(b, p, br, pr), (nb, np_)


def test_capacity_error_reports_required_count():
    b = np.arange(1000, dtype=np.int32)
    p = np.tile(np.arange(1000, dtype=np.int32), 3)
    j = api.Joiner(dev(b), dev(p), True, capacity=10)
    j.launch()
    with pytest.raises(PJError) as e:
        j.result()
    assert int(j.count.item()) == 3000
    assert "capacity" in str(e.value)


@pytest.mark.parametrize("pdtype", [np.int32, np.int64, np.float32])
@pytest.mark.parametrize("unique", [True, False])
def test_join_payload_gather(pdtype, unique):
    rng = np.random.default_rng(24)
    b = rng.permutation(300000).astype(np.int32)
    if not unique:
        b = np.concatenate([b, b[:20000]])
    p = rng.integers(0, 400000, size=500000).astype(np.int32)
    bp = (rng.standard_normal(b.shape[0]) * 1000).astype(pdtype)
    pp = (rng.standard_normal(p.shape[0]) * 1000).astype(pdtype)
    br, pr, gb, gp = api.partitioned_join_payload(dev(b), dev(p), dev(bp), dev(pp), unique_build_keys=unique)
    br, pr = br.cpu().numpy(), pr.cpu().numpy()
    assert np.array_equal(gb.cpu().numpy(), bp[br])
    assert np.array_equal(gp.cpu().numpy(), pp[pr])
    assert pairs_equal(b, p, torch.from_numpy(br), torch.from_numpy(pr), unique)
    # one side only
    _, pr2, none_b, gp2 = api.partitioned_join_payload(dev(b), dev(p), None, dev(pp), unique_build_keys=unique)
    assert none_b is None and np.array_equal(gp2.cpu().numpy(), pp[pr2.cpu().numpy()])


def test_join_count_matches_oracle():
    b, p = datagen.config2(seed=17, n_build=100000, n_probe=200000)
    assert api.join_count(dev(b), dev(p)) == oracle.inner_join(b, p)[0].shape[0]


def test_misaligned_input_rejected():
    b = dev(np.arange(101, dtype=np.int32))
    p = dev(np.arange(100, dtype=np.int32))
    with pytest.raises(PJError) as e:
        api.partitioned_join(b[1:], p)
    assert e.value.status == 7
