"""The heavy-key path: heavy probe keys (named by the plan) bypass the
partitions and are matched by a table every CTA holds.  The output must be
the oracle's multiset whatever the heavy set holds: keys with a build row,
keys without one, keys that never occur, and outputs past the capacity."""
import numpy as np
import pytest
import torch

from oracle import oracle
from partitioned_join_b200 import PJError, api, datagen

pytestmark = pytest.mark.gpu


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def check_pairs(b, p, br, pr, unique=True):
    eb, ep = oracle.inner_join(b, p, unique)
    got = oracle.sorted_pairs(br.cpu().numpy(), pr.cpu().numpy())
    exp = oracle.sorted_pairs(eb, ep)
    assert got.shape == exp.shape and np.array_equal(got, exp)


@pytest.mark.parametrize("theta", [1.0, 1.5])
def test_exact_planner_finds_heavy_keys_and_joins_exactly(theta):
    b, p = datagen.config3(seed=51, theta=theta, n_build=1 << 18, n_probe=1 << 21)
    bt, pt = dev(b), dev(p)
    plan = api.plan_exact(bt, pt, True)
    assert plan.n_heavy > 0 or theta < 1.25
    # the named keys are the most frequent probe keys
    vals, counts = np.unique(p, return_counts=True)
    top = set(vals[np.argsort(-counts)[: plan.n_heavy // 2]].tolist())
    assert top <= set(plan.as_dict()["heavy_keys"])
    br, pr = api.partitioned_join(bt, pt, plan=plan)
    check_pairs(b, p, br, pr)


@pytest.mark.parametrize("dtype", [np.int32, np.int64])
def test_heavy_keys_with_and_without_build_rows(dtype):
    rng = np.random.default_rng(52)
    b = rng.permutation(400000).astype(dtype)
    p = np.concatenate([rng.integers(0, 500000, size=600000), np.full(200000, 17), np.full(150000, 450001),
                        np.full(50000, -5)]).astype(dtype)
    rng.shuffle(p)
    bt, pt = dev(b), dev(p)
    plan = api.plan_default(b.shape[0], p.shape[0], np.dtype(dtype).itemsize)
    # 17: in the build side; 450001, -5: not; 123456789: never probed
    plan.set_heavy([17, 450001, -5, 123456789] + list(range(1000, 1100)))
    br, pr = api.partitioned_join(bt, pt, plan=plan)
    check_pairs(b, p, br, pr)
    assert api.join_count(bt, pt, plan=plan) == br.numel()


def test_heavy_outputs_past_capacity_report_the_count():
    b = np.arange(1000, dtype=np.int32)
    p = np.concatenate([np.full(5000, 7, np.int32), np.arange(1000, dtype=np.int32)])
    plan = api.plan_default(b.shape[0], p.shape[0], 4)
    plan.set_heavy([7])
    j = api.Joiner(dev(b), dev(p), True, plan, capacity=100)
    j.launch()
    with pytest.raises(PJError):
        j.result()
    assert int(j.count.item()) == 6000
    br, pr = api.partitioned_join(dev(b), dev(p), plan=plan)   # grows the output and reruns
    check_pairs(b, p, br, pr)


def test_heavy_plan_ignored_for_repeated_build_keys():
    rng = np.random.default_rng(53)
    b = rng.integers(0, 50000, size=200000).astype(np.int32)
    p = np.concatenate([rng.integers(0, 60000, size=300000), np.full(100000, 42)]).astype(np.int32)
    plan = api.plan_default(b.shape[0], p.shape[0], 4, False)
    plan.set_heavy([42])
    br, pr = api.partitioned_join(dev(b), dev(p), unique_build_keys=False, plan=plan)
    check_pairs(b, p, br, pr, unique=False)


def test_uniform_probe_names_no_heavy_keys():
    b, p = datagen.config2(seed=54, n_build=1 << 20, n_probe=1 << 21)
    assert api.plan_exact(dev(b), dev(p), True).n_heavy == 0
