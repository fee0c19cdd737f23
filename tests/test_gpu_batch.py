"""Batches of joins (pj_join_batch): every join's pairs must equal the
oracle's, whichever path (direct table or partitioned) it takes, in a plain
launch, in CUDA graph replays, and after the autotuner has picked a
configuration."""
import numpy as np
import pytest
import torch

from oracle import oracle
from partitioned_join_b200 import api

pytestmark = pytest.mark.gpu


def _batch(seed, n, dtype=torch.int32, lo=0, hi=17, unique=True):
    rng = np.random.default_rng(seed)
    pairs, host = [], []
    for i in range(n):
        nb = int(2 ** rng.uniform(lo, hi))
        np_ = int(nb * rng.choice([1, 4])) + int(rng.integers(0, 5))
        theta = 1.0 if i % 4 == 0 else 0.0
        b, p, _ = api.generate_tables(nb, np_, dtype, rand_max=max(nb - 1, 0) if unique else max(nb // 3, 1),
                                      selectivity=0.7, unique_build_keys=unique, zipf_theta=theta,
                                      seed=seed * 1000 + i)
        pairs.append((b, p))
        host.append((b.cpu().numpy(), p.cpu().numpy()))
    return pairs, host


def _check(bj, host, unique=True):
    for (br, pr), (b, p) in zip(bj.results(), host):
        eb, ep = oracle.inner_join(b, p, unique)
        got = oracle.sorted_pairs(br.cpu().numpy(), pr.cpu().numpy())
        assert np.array_equal(got, oracle.sorted_pairs(eb, ep))


@pytest.mark.parametrize("dtype", [torch.int32, torch.int64])
def test_batch_matches_oracle(dtype):
    pairs, host = _batch(61, 40, dtype)
    bj = api.BatchJoiner(pairs)
    bj.launch()
    _check(bj, host)


def test_batch_repeated_build_keys():
    pairs, host = _batch(62, 16, torch.int32, 4, 15, unique=False)
    bj = api.BatchJoiner(pairs, unique_build_keys=False)
    bj.launch()
    _check(bj, host, unique=False)


def test_batch_edge_sizes():
    # empty sides, a single row, all-direct and all-partitioned limits
    sizes = [(0, 10), (10, 0), (1, 1), (3, 1000), (20480, 5), (20481, 100000), (1 << 17, 1 << 16)]
    pairs, host = [], []
    for i, (nb, np_) in enumerate(sizes):
        b, p, _ = api.generate_tables(nb, np_, torch.int32, max(nb * 2, 1), 0.8, True, 0.0, 70 + i)
        pairs.append((b, p))
        host.append((b.cpu().numpy(), p.cpu().numpy()))
    for limit in (0, 20480):
        bj = api.BatchJoiner(pairs)
        bj.config.direct_max_build = limit
        bj.prepare()
        bj.launch()
        _check(bj, host)


def test_batch_graph_replay():
    pairs, host = _batch(63, 24)
    bj = api.BatchJoiner(pairs)
    g = bj.graph()
    for _ in range(2):
        bj.count.zero_()
        g.replay()
        torch.cuda.synchronize()
        _check(bj, host)


def test_batch_autotune_keeps_results():
    pairs, host = _batch(64, 24)
    bj = api.BatchJoiner(pairs)
    ms = bj.autotune()
    assert ms > 0
    c = bj.config.as_dict()
    assert c["direct_threads"] in (256, 512, 1024) and 0 <= c["direct_max_build"] <= 40960
    bj.launch()
    _check(bj, host)


@pytest.mark.parametrize("dtype", [torch.int32, torch.int64])
def test_batch_large_joins_run_together(dtype):
    # joins of 2^18..2^20 build rows: partitioned by one histogram, scan and
    # scatter launch over all of them and joined by one persistent launch;
    # the same batch run one join after another must give the same pairs
    pairs, host = _batch(65, 10, dtype, 18, 20)
    for together in (1, 0):
        bj = api.BatchJoiner(pairs)
        bj.config.large_batched = together
        bj.prepare()
        bj.launch()
        _check(bj, host)


def test_batch_large_joins_repeated_keys_and_graph():
    pairs, host = _batch(66, 12, torch.int32, 15, 18, unique=False)
    bj = api.BatchJoiner(pairs, unique_build_keys=False)
    bj.config.direct_max_build = 0  # every join partitioned, all together
    bj.prepare()
    g = bj.graph()
    for _ in range(2):
        g.replay()
        torch.cuda.synchronize()
        _check(bj, host, unique=False)
