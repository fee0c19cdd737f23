"""The learned planner: its network's CUDA forward/backward/Adam kernels
against the float64 oracle (oracle/mlp_oracle.py), training that lowers the
loss, and joins under learned plans that stay bit-exact -- including a plan
that overflows on the device and falls back to the exact planner."""
import ctypes

import numpy as np
import pytest
import torch

from oracle import mlp_oracle, oracle
from partitioned_join_b200 import _lib, api, datagen, planner

pytestmark = pytest.mark.gpu

D = (_lib.MLP_FEATURES, _lib.MLP_HIDDEN, _lib.MLP_HIDDEN, _lib.PLAN_CANDIDATES)


def _rand(seed, batch=37):
    rng = np.random.default_rng(seed)
    params = rng.normal(0, 0.2, planner.N_PARAMS).astype(np.float32)
    x = rng.normal(0, 1, (batch, D[0])).astype(np.float32)
    dy = rng.normal(0, 1, (batch, D[3])).astype(np.float32)
    return params, x, dy


def test_forward_and_gradients_match_the_oracle():
    params, x, dy = _rand(81)
    net = planner.Mlp(torch.from_numpy(params))
    xd = torch.from_numpy(x).cuda()
    y, acts = net.forward(xd)
    grad = net.backward(xd, acts, torch.from_numpy(dy).cuda())
    ey, cache = mlp_oracle.forward(params, x, *D)
    eg = mlp_oracle.backward(params, cache, dy, *D)
    np.testing.assert_allclose(y.cpu().numpy(), ey, rtol=1e-4, atol=1e-4)
    np.testing.assert_allclose(grad.cpu().numpy(), eg, rtol=1e-3, atol=2e-4)


def test_gradient_matches_finite_differences_of_the_oracle():
    # the oracle's own chain rule, checked numerically on a few weights
    params, x, dy = _rand(82, batch=5)
    p64 = params.astype(np.float64)
    _, cache = mlp_oracle.forward(p64, x, *D)
    g = mlp_oracle.backward(p64, cache, dy, *D)
    rng = np.random.default_rng(3)
    for i in rng.choice(p64.shape[0], 12, replace=False):
        e = np.zeros_like(p64)
        e[i] = 1e-6
        f = lambda q: float((mlp_oracle.forward(q, x, *D)[0] * dy).sum())  # noqa: E731
        num = (f(p64 + e) - f(p64 - e)) / 2e-6
        assert abs(num - g[i]) < 1e-4 * max(1.0, abs(num))


def test_mse_and_adam_match_the_oracle():
    rng = np.random.default_rng(83)
    y = rng.normal(size=(40, 12)).astype(np.float32)
    t = rng.normal(size=(40, 12)).astype(np.float32)
    m = (rng.random((40, 12)) < 0.7).astype(np.float32)
    yd, td, md = (torch.from_numpy(a).cuda() for a in (y, t, m))
    dy = torch.empty_like(yd)
    loss = torch.zeros(1, device="cuda")
    L = _lib.lib()
    _lib.check(L.pj_mlp_mse_grad(ctypes.c_void_p(yd.data_ptr()), ctypes.c_void_p(td.data_ptr()),
                                 ctypes.c_void_p(md.data_ptr()), y.size, ctypes.c_void_p(dy.data_ptr()),
                                 ctypes.c_void_p(loss.data_ptr()), None))
    edy, eloss = mlp_oracle.mse_grad(y, t, m)
    np.testing.assert_allclose(dy.cpu().numpy(), edy, rtol=1e-5, atol=1e-7)
    assert abs(float(loss.item()) - eloss) < 1e-4 * max(1, eloss)
    p = rng.normal(size=1000).astype(np.float32)
    g = rng.normal(size=1000).astype(np.float32)
    pd, gd = torch.from_numpy(p).cuda(), torch.from_numpy(g).cuda()
    md, vd = torch.zeros_like(pd), torch.zeros_like(pd)
    ep, em, ev = p.astype(np.float64), np.zeros(1000), np.zeros(1000)
    for step in (1, 2, 3):
        _lib.check(L.pj_mlp_adam(ctypes.c_void_p(pd.data_ptr()), ctypes.c_void_p(gd.data_ptr()),
                                 ctypes.c_void_p(md.data_ptr()), ctypes.c_void_p(vd.data_ptr()), 1000, 1e-2, 0.9,
                                 0.999, 1e-8, step, None))
        ep, em, ev = mlp_oracle.adam(ep, g, em, ev, 1e-2, 0.9, 0.999, 1e-8, step)
    np.testing.assert_allclose(pd.cpu().numpy(), ep, rtol=1e-5, atol=1e-6)


def test_training_fits_a_teacher_network():
    rng = np.random.default_rng(84)
    teacher = planner.Mlp(torch.from_numpy(rng.normal(0, 0.3, planner.N_PARAMS).astype(np.float32)))
    X = rng.normal(size=(2000, D[0])).astype(np.float32)
    T = teacher.predict(X)
    M = np.ones_like(T)
    student = planner.Mlp(seed=5)
    losses = student.train(X, T, M, steps=2000, lr=3e-3)
    assert losses[-1] < 0.25 * losses[0]


def test_features_are_a_function_of_the_probe_sample():
    b, p = datagen.config3(seed=85, theta=1.5, n_build=1 << 16, n_probe=1 << 20)
    f1, heavy = planner.features(torch.from_numpy(b).cuda(), torch.from_numpy(p).cuda())
    b2, p2 = datagen.config2(seed=86, n_build=1 << 16, n_probe=1 << 20)
    f2, heavy2 = planner.features(torch.from_numpy(b2).cuda(), torch.from_numpy(p2).cuda())
    assert f1.shape == (D[0],) and np.all(np.isfinite(f1))
    assert f1[0] > f2[0]                 # the skewed sample has a heavier top bin
    assert heavy.n_heavy > 0 and heavy2.n_heavy == 0


@pytest.mark.parametrize("case", ["uniform32", "zipf64"])
def test_learned_plans_join_exactly(case):
    if case == "uniform32":
        b, p = datagen.config2(seed=87, n_build=1 << 20, n_probe=1 << 21)
    else:
        b, p = datagen.config3(seed=88, theta=1.25, n_build=1 << 17, n_probe=1 << 21)
    bt, pt = torch.from_numpy(b).cuda(), torch.from_numpy(p).cuda()
    for seed in (1, 2):
        params = planner.Mlp(seed=seed).params
        br, pr, info = planner.partitioned_join_learned(bt, pt, True, params)
        eb, ep = oracle.inner_join(b, p, True)
        assert np.array_equal(oracle.sorted_pairs(br.cpu().numpy(), pr.cpu().numpy()), oracle.sorted_pairs(eb, ep))


def test_overflowing_choice_falls_back_to_the_exact_plan():
    # weights that always rank candidate 9 (COMPACT tables, one radix bit
    # fewer, no heavy keys) first: at 2^21 build rows its partitions exceed a
    # COMPACT entry's 16-bit index range and the device reports an overflow
    w = np.zeros(planner.N_PARAMS, dtype=np.float32)
    bias = w[-_lib.PLAN_CANDIDATES:]
    bias[:] = 10.0
    bias[9] = -10.0
    b, p = datagen.config2(seed=89, n_build=1 << 21, n_probe=1 << 21)
    bt, pt = torch.from_numpy(b).cuda(), torch.from_numpy(p).cuda()
    plan, scores = planner.plan_learned(bt, pt, True, torch.from_numpy(w).cuda())
    assert int(np.argmin(scores)) == 9 and plan.table_mode == _lib.TABLE_COMPACT
    br, pr, info = planner.partitioned_join_learned(bt, pt, True, torch.from_numpy(w).cuda())
    assert info["fallback"]
    eb, ep = oracle.inner_join(b, p, True)
    assert np.array_equal(oracle.sorted_pairs(br.cpu().numpy(), pr.cpu().numpy()), oracle.sorted_pairs(eb, ep))


def test_shipped_weights_gain_over_exact_plans():
    """What the trained network gains: on a small seeded set of joins it was
    not trained on (build 2^20..2^24 rows, probe 1/4/16x, int32/int64, Zipf
    0..1.5, match 0.1..1), the joins under the shipped network's plans take
    less time in total (geometric mean of the per-join speedups) than under
    the exact-histogram planner's, a fallback counted at its full cost, and
    give the same pairs."""
    params = planner.load_weights()
    assert params is not None, "shipped weights missing"
    rng = np.random.default_rng(20261203)
    speed = []
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def best_ms(j):
        j.launch()
        st = j.status()
        t = float("inf")
        for _ in range(3):
            e0.record()
            j.launch()
            e1.record()
            torch.cuda.synchronize()
            t = min(t, e0.elapsed_time(e1))
        return t, st

    for _ in range(20):
        b, p, meta = planner.sweep_workload(rng, 24, 26, min_log2_build=20)
        exact = api.plan_exact(b, p, True)
        t_exact, st = best_ms(api.Joiner(b, p, True, exact))
        assert st == _lib.OK
        learned, _ = planner.plan_learned(b, p, True, params)
        jl = api.Joiner(b, p, True, learned)
        t_learned, st = best_ms(jl)
        if st != _lib.OK:
            t_learned += t_exact  # the fallback reruns the exact plan
        else:
            n = int(jl.count.item())
            ref = api.Joiner(b, p, True, exact)
            ref.launch()
            rb, rp = ref.result()
            assert n == rb.shape[0]
            got = torch.sort(jl.probe_row[:n].long() * b.numel() + jl.build_row[:n].long())[0]
            exp = torch.sort(rp.long() * b.numel() + rb.long())[0]
            assert torch.equal(got, exp)
        speed.append(t_exact / t_learned)
        del b, p
    geo = float(np.exp(np.mean(np.log(speed))))
    assert geo > 1.0, (geo, speed)
