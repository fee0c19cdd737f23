"""Device input generation (pj_generate_tables): the reference's table
recipe (generate_input_tables.cuh:35-226) and Zipf probe keys
(generate_zipf_input.cuh:21-134), checked for the properties the joins rely
on: distinct build keys in range, hits exactly the probe keys present in
the build side, determinism per seed, and the Zipf rank frequencies."""
import numpy as np
import pytest
import torch

from partitioned_join_b200 import api

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", [torch.int32, torch.int64])
@pytest.mark.parametrize("rand_max_factor", [1, 3])
def test_unique_build_and_selectivity(dtype, rand_max_factor):
    nb, np_ = 1 << 20, 1 << 21
    rmax = nb * rand_max_factor - 1
    b, p, hits = api.generate_tables(nb, np_, dtype, rmax, selectivity=0.7, seed=5)
    bn, pn = b.cpu().numpy(), p.cpu().numpy()
    assert np.unique(bn).shape[0] == nb and bn.min() >= 0 and bn.max() <= rmax
    present = np.isin(pn, bn)
    assert present.sum() == hits                              # misses never hit the build side
    assert abs(hits / np_ - 0.7) < 0.005
    if rand_max_factor == 1:
        assert np.all(pn[~present] > rmax)                    # domain used up: misses above it
    else:
        assert np.all((pn[~present] >= 0) & (pn[~present] <= rmax))


def test_repeated_build_keys_in_range():
    b, p, hits = api.generate_tables(1 << 18, 1 << 18, torch.int32, 1000, selectivity=0.5, unique_build_keys=False,
                                     seed=6)
    bn = b.cpu().numpy()
    assert bn.min() >= 0 and bn.max() <= 1000 and np.unique(bn).shape[0] <= 1001
    assert abs(hits / (1 << 18) - 0.5) < 0.01


def test_deterministic_per_seed():
    a = api.generate_tables(100000, 300000, torch.int32, 500000, 0.9, seed=7)
    b = api.generate_tables(100000, 300000, torch.int32, 500000, 0.9, seed=7)
    c = api.generate_tables(100000, 300000, torch.int32, 500000, 0.9, seed=8)
    assert torch.equal(a[0], b[0]) and torch.equal(a[1], b[1]) and a[2] == b[2]
    assert not torch.equal(a[0], c[0])


@pytest.mark.parametrize("theta", [0.5, 1.0, 1.5])
def test_zipf_rank_frequencies(theta):
    nb, np_ = 1 << 16, 1 << 22
    _, p, hits = api.generate_tables(nb, np_, torch.int32, selectivity=1.0, zipf_theta=theta, seed=9)
    assert hits == np_
    counts = np.sort(np.bincount(p.cpu().numpy(), minlength=nb))[::-1].astype(np.float64)
    w = 1.0 / np.power(np.arange(1, nb + 1, dtype=np.float64), theta)
    pmf = w / w.sum()
    # the heaviest ranks: within 5 sigma of their binomial expectation
    for r in range(8):
        e = np_ * pmf[r]
        assert abs(counts[r] - e) < 5 * np.sqrt(e * (1 - pmf[r])) + 1, (r, counts[r], e)
    # the mass of the first 1 % of ranks
    k = nb // 100
    assert abs(counts[:k].sum() / np_ - pmf[:k].sum()) < 0.01
