"""Pair-level parity at the benchmark configurations' own sizes.

The reference checks every run against inner_join_cpu (main.cu:910-916,
inner_join_cpu.hpp:110-168).  These tests do the same at the sizes the bench
runs, against the C restatement of inner_join_cpu (oracle.inner_join):

* cfg1 at exactly 2^20 x 2^22 (int32, 100 % matches);
* cfg2 at 2^27 x 2^27 (int32, 90 % matches) under the plan the bench runs:
  one pass of 12 hash-digit bits, EXACT tables of 2^15 buckets whose
  entries hold 5 tag bits above 27 build-row bits -- the only size at which
  that bit budget occurs;
* cfg3 at 2^24 x 2^26 (int64) with Zipf 1.5 probe keys (heavy-key path) and
  Zipf 0;
* cfg5: a whole 512-join batch.

With unique build keys every probe row matches at most once, so two outputs
are the same multiset exactly when they give every probe row the same build
row (or none); `same_pairs` compares them that way in O(n).
"""
import numpy as np
import pytest
import torch

from oracle import oracle
from partitioned_join_b200 import DIGIT_HASH, TABLE_EXACT, api, datagen

pytestmark = pytest.mark.gpu

DEV = "cuda:0"


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def partner_of(build_row, probe_row, n_probe):
    """Build row of every probe row (-1: unmatched); None if a probe row
    appears twice (impossible for a unique-key join)."""
    part = np.full(n_probe, -1, dtype=np.int64)
    if probe_row.shape[0] and np.bincount(probe_row, minlength=n_probe).max() > 1:
        return None
    part[probe_row] = build_row
    return part


def same_pairs(b, p, got_b, got_p):
    eb, ep = oracle.inner_join(b, p, True)
    assert eb.shape[0] == got_b.shape[0], (eb.shape[0], got_b.shape[0])
    exp = partner_of(eb.astype(np.int64), ep.astype(np.int64), p.shape[0])
    got = partner_of(got_b.astype(np.int64), got_p.astype(np.int64), p.shape[0])
    assert exp is not None and got is not None
    return np.array_equal(exp, got)


def test_cfg1_full_size_matches_oracle():
    b, p = datagen.config1(seed=11)
    assert b.shape[0] == 1 << 20 and p.shape[0] == 1 << 22
    db, dp = dev(b), dev(p)
    for plan in (None, api.plan_exact(db, dp, True)):
        br, pr = api.partitioned_join(db, dp, True, plan=plan)
        assert same_pairs(b, p, br.cpu().numpy(), pr.cpu().numpy())


def test_cfg2_headline_plan_full_size_matches_oracle():
    n = 1 << 27
    db, dp, hits = api.generate_tables(n, n, torch.int32, n - 1, 0.9, True, 0.0, 2, DEV)
    plan = api.plan_default(n, n, 4, True)
    # the bench's plan: 4096 partitions by hash bits, EXACT tables, 2^15
    # buckets; an entry keeps 32 - 12 - 15 = 5 tag bits above 27 row bits
    assert (plan.passes, plan.bits1, plan.digit_mode, plan.table_mode) == (1, 12, DIGIT_HASH, TABLE_EXACT)
    assert plan.as_dict() == api.plan_exact(db, dp, True).as_dict()
    j = api.Joiner(db, dp, True, plan, capacity=n)
    j.launch()
    br, pr = j.result()
    assert br.shape[0] == hits
    got_b, got_p = br.cpu().numpy(), pr.cpu().numpy()
    del br, pr, j
    b, p = db.cpu().numpy(), dp.cpu().numpy()
    del db, dp
    torch.cuda.empty_cache()
    assert same_pairs(b, p, got_b, got_p)


@pytest.mark.parametrize("theta", [1.5, 0.0])
def test_cfg3_int64_zipf_matches_oracle(theta):
    nb, np_ = 1 << 24, 1 << 26
    db, dp, hits = api.generate_tables(nb, np_, torch.int64, (1 << 62) - 1, 1.0, True, theta, 3, DEV)
    plan = api.plan_exact(db, dp, True)
    if theta == 1.5:
        assert plan.n_heavy > 0  # the heavy-key broadcast-probe path runs
    br, pr = api.partitioned_join(db, dp, True, plan=plan)
    assert br.shape[0] == hits == np_
    assert same_pairs(db.cpu().numpy(), dp.cpu().numpy(), br.cpu().numpy(), pr.cpu().numpy())


def test_cfg5_full_batch_matches_oracle():
    rng = np.random.default_rng(5)
    pairs = []
    for i in range(512):
        nb = int(2 ** rng.uniform(10, 20))
        b, p, _ = api.generate_tables(nb, 4 * nb, torch.int32, nb - 1, 0.7, True, 1.0 if i % 4 == 3 else 0.0,
                                      9000 + i, DEV)
        pairs.append((b, p))
    bj = api.BatchJoiner(pairs)
    bj.launch()
    for (br, pr), (b, p) in zip(bj.results(), pairs):
        assert same_pairs(b.cpu().numpy(), p.cpu().numpy(), br.cpu().numpy(), pr.cpu().numpy())
