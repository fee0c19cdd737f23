"""Learned planner: an MLP that ranks candidate schedules of a join.

The network (PJ_MLP_FEATURES -> 64 -> 64 -> PJ_PLAN_CANDIDATES, ~8 K FP32
weights) reads a sketch of a probe-key sample plus the sizes
(pj_plan_features) and predicts, for each candidate schedule (one pass with
BUCKET, COMPACT or EXACT tables x radix bits x heavy-key set, or two passes,
pj_plan_candidate), its run time relative to the others (log2 ms minus the
workload's mean).  It is trained on the GPU by
the library's own kernels (pj_mlp_forward / pj_mlp_backward /
pj_mlp_mse_grad / pj_mlp_adam) on timings that the plain method generates
over a seeded synthetic sweep.  The exact-histogram planner (pj_plan_exact)
is both the fallback -- a learned choice whose table overflows on the device
is rerun with it -- and the yardstick: the sweep times it beside every
candidate.  The network picks a schedule, never a result.

    python -m partitioned_join_b200.planner --train --workloads 400 --out weights.npz

The reference has no planner of this kind (its -n/-N/-f flags fix the
schedule, main.cu:100-188).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import time
from typing import List, Optional

import numpy as np
import torch

from . import _lib, api
from ._lib import JoinDesc, MlpDims, Output, Plan, check, lib

PKG = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(PKG, "planner_weights.npz")
DIMS = MlpDims(_lib.MLP_FEATURES, _lib.MLP_HIDDEN, _lib.MLP_HIDDEN, _lib.PLAN_CANDIDATES)
N_PARAMS = _lib.MLP_FEATURES * 64 + 64 + 64 * 64 + 64 + 64 * _lib.PLAN_CANDIDATES + _lib.PLAN_CANDIDATES


def _p(t: torch.Tensor):
    return ctypes.c_void_p(t.data_ptr())


def _st():
    return api._stream_ptr(None)


class Mlp:
    """The network's parameters on the device and its training loop, every
    step in the library's kernels."""

    def __init__(self, params: Optional[torch.Tensor] = None, seed: int = 0, device="cuda"):
        assert lib().pj_mlp_param_count(ctypes.byref(DIMS)) == N_PARAMS
        if params is None:
            g = np.random.default_rng(seed)
            parts = []
            for fan_in, fan_out in ((DIMS.in_, DIMS.h1), (DIMS.h1, DIMS.h2), (DIMS.h2, DIMS.out)):
                lim = math.sqrt(6.0 / fan_in)  # He-uniform for ReLU layers
                parts += [g.uniform(-lim, lim, size=fan_in * fan_out), np.zeros(fan_out)]
            params = torch.from_numpy(np.concatenate(parts).astype(np.float32))
        self.params = params.to(device=device, dtype=torch.float32).contiguous()
        self.device = self.params.device

    def forward(self, x: torch.Tensor):
        b = x.shape[0]
        acts = torch.empty(b, 2 * DIMS.h1 + 2 * DIMS.h2, dtype=torch.float32, device=self.device)
        y = torch.empty(b, DIMS.out, dtype=torch.float32, device=self.device)
        check(lib().pj_mlp_forward(_p(self.params), ctypes.byref(DIMS), _p(x), b, _p(acts), _p(y), _st()),
              "pj_mlp_forward")
        return y, acts

    def backward(self, x, acts, dy) -> torch.Tensor:
        b = x.shape[0]
        grad = torch.empty_like(self.params)
        scratch = torch.empty(b, DIMS.h1 + DIMS.h2, dtype=torch.float32, device=self.device)
        check(lib().pj_mlp_backward(_p(self.params), ctypes.byref(DIMS), _p(x), _p(acts), _p(dy), b, _p(grad),
                                    _p(scratch), _st()), "pj_mlp_backward")
        return grad

    def train(self, X, T, M, steps=2000, lr=3e-3, batch=256, seed=0) -> List[float]:
        X, T, M = (torch.as_tensor(a, dtype=torch.float32, device=self.device).contiguous() for a in (X, T, M))
        m = torch.zeros_like(self.params)
        v = torch.zeros_like(self.params)
        loss = torch.zeros(1, dtype=torch.float32, device=self.device)
        g = torch.Generator(device="cpu").manual_seed(seed)
        losses = []
        n = X.shape[0]
        for step in range(1, steps + 1):
            idx = torch.randint(0, n, (min(batch, n),), generator=g).to(self.device)
            xb, tb, mb = X[idx].contiguous(), T[idx].contiguous(), M[idx].contiguous()
            y, acts = self.forward(xb)
            dy = torch.empty_like(y)
            check(lib().pj_mlp_mse_grad(_p(y), _p(tb), _p(mb), y.numel(), _p(dy), _p(loss), _st()), "pj_mlp_mse_grad")
            grad = self.backward(xb, acts, dy)
            check(lib().pj_mlp_adam(_p(self.params), _p(grad), _p(m), _p(v), self.params.numel(), lr, 0.9, 0.999,
                                    1e-8, step, _st()), "pj_mlp_adam")
            if step % 50 == 0 or step == steps:
                losses.append(float(loss.item()))
        return losses

    def predict(self, X) -> np.ndarray:
        x = torch.as_tensor(X, dtype=torch.float32, device=self.device).contiguous()
        return self.forward(x)[0].cpu().numpy()


def load_weights(path: str = WEIGHTS, device="cuda") -> Optional[torch.Tensor]:
    if not os.path.exists(path):
        return None
    w = np.load(path)["params"].astype(np.float32)
    if w.shape[0] != N_PARAMS:
        raise ValueError(f"{path}: {w.shape[0]} parameters, expected {N_PARAMS}")
    return torch.from_numpy(w).to(device)


# ---------------------------------------------------------------------------
# planning and joining with the network

def _ws_for(desc: JoinDesc, plans) -> int:
    return max(api.workspace_size(desc, p) for p in plans)


def features(build, probe, unique=True):
    """(features[PJ_MLP_FEATURES], heavy-set plan) of a join."""
    d = api.make_desc(build, probe, unique)
    base = api.plan_default(d.n_build, d.n_probe, d.key_bytes, unique)
    nb = api.workspace_size(d, base)
    ws = api.alloc_workspace(nb, build.device)
    f = (ctypes.c_float * _lib.MLP_FEATURES)()
    heavy = Plan()
    check(lib().pj_plan_features(ctypes.byref(d), _p(ws), nb, f, ctypes.byref(heavy), _st()), "pj_plan_features")
    return np.array(list(f), dtype=np.float32), heavy


def candidate(build, probe, c: int, heavy: Plan, unique=True) -> Optional[Plan]:
    d = api.make_desc(build, probe, unique)
    p = Plan()
    st = lib().pj_plan_candidate(ctypes.byref(d), c, ctypes.byref(heavy), ctypes.byref(p))
    return p if st == _lib.OK else None


def plan_learned(build, probe, unique=True, params: Optional[torch.Tensor] = None,
                 ws: Optional[torch.Tensor] = None):
    """(plan, scores) from the network (default: the shipped weights).  ws:
    a workspace of at least the default plan's size to reuse."""
    if params is None:
        params = load_weights(device=build.device)
        if params is None:
            raise RuntimeError(f"no planner weights at {WEIGHTS}: train them first")
    d = api.make_desc(build, probe, unique)
    base = api.plan_default(d.n_build, d.n_probe, d.key_bytes, unique)
    nb = api.workspace_size(d, base)
    if ws is None or ws.numel() < nb:
        ws = api.alloc_workspace(nb, build.device)
    p = Plan()
    scores = (ctypes.c_float * _lib.PLAN_CANDIDATES)()
    check(lib().pj_plan_learned(ctypes.byref(d), _p(params), _p(ws), nb, ctypes.byref(p), scores, _st()),
          "pj_plan_learned")
    return p, np.array(list(scores), dtype=np.float32)


def partitioned_join_learned(build, probe, unique=True, params: Optional[torch.Tensor] = None):
    """The join under the learned plan; a plan whose table overflows on the
    device is replaced by the exact planner's.  Returns (build_row,
    probe_row, info) with info = {"fallback": bool, "plan": dict}."""
    plan, _ = plan_learned(build, probe, unique, params)
    j = api.Joiner(build, probe, unique, plan)
    j.launch()
    st = j.status()
    if st == _lib.OK:
        n = int(j.count.item())
        return j.build_row[:n], j.probe_row[:n], {"fallback": False, "plan": plan.as_dict()}
    if st not in (_lib.ERR_OVERFLOW, _lib.ERR_INTERNAL, _lib.ERR_CAPACITY):
        check(st, "pj_inner_join")
    exact = api.plan_exact(build, probe, unique)
    br, pr = api.partitioned_join(build, probe, unique, exact)
    return br, pr, {"fallback": st != _lib.ERR_CAPACITY, "plan": exact.as_dict()}


# ---------------------------------------------------------------------------
# training data: a seeded sweep timed by the plain method

def _time_join(desc, plan, ws, nb, out, reps=2) -> (float, int):
    L = lib()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    L.pj_inner_join(ctypes.byref(desc), ctypes.byref(plan), ctypes.byref(out), _p(ws), nb, _st())
    status = L.pj_check(_p(ws), _st())
    best = float("inf")
    for _ in range(reps):
        e0.record()
        L.pj_inner_join(ctypes.byref(desc), ctypes.byref(plan), ctypes.byref(out), _p(ws), nb, _st())
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
        status = status or L.pj_check(_p(ws), _st())
    return best, status


def sweep_workload(rng: np.random.Generator, max_log2_build=28, max_log2_probe=29, device="cuda",
                   min_log2_build=18):
    """One seeded workload of the planner sweep: build rows log-uniform in
    2^min..2^max, probe/build ratio 1, 4 or 16 (the probe side capped at
    2^max_log2_probe rows: row ids are int32, and a 2^28 x 2^32 join would
    need about 100 GB of workspace), int32 or int64 keys, Zipf exponent
    uniform in [0, 1.5] (0 below 0.2), match rate in [0.1, 1]."""
    lb = rng.uniform(min_log2_build, max_log2_build)
    nb = int(2 ** lb)
    ratio = int(rng.choice([1, 4, 16]))
    np_ = min(nb * ratio, 1 << max_log2_probe)
    dtype = torch.int32 if rng.random() < 0.5 else torch.int64
    theta = float(rng.uniform(0, 1.5))
    theta = 0.0 if theta < 0.2 else theta
    match = float(rng.uniform(0.1, 1.0))
    rand_max = nb - 1 if dtype == torch.int32 else (1 << 40)
    b, p, _ = api.generate_tables(nb, np_, dtype, rand_max, match, True, theta, int(rng.integers(1 << 62)), device)
    return b, p, {"n_build": nb, "n_probe": np_, "key_bytes": 4 if dtype == torch.int32 else 8, "zipf": theta,
                  "match": match}


def measure(build, probe):
    """Features and the time of every candidate and of the exact plan."""
    feat, heavy = features(build, probe)
    d = api.make_desc(build, probe, True)
    cands = [candidate(build, probe, c, heavy) for c in range(_lib.PLAN_CANDIDATES)]
    exact = api.plan_exact(build, probe, True)
    cands[_lib.PLAN_CANDIDATE_EXACT] = None  # timed below as the exact plan
    plans = [p for p in cands if p is not None] + [exact]
    nb = _ws_for(d, plans)
    ws = api.alloc_workspace(nb, build.device)
    cap = probe.numel()
    br = torch.empty(max(cap, 1), dtype=torch.int32, device=build.device)
    pr = torch.empty_like(br)
    cnt = torch.zeros(1, dtype=torch.int64, device=build.device)
    out = Output()
    out.build_row, out.probe_row, out.capacity, out.count = br.data_ptr(), pr.data_ptr(), cap, cnt.data_ptr()
    times = np.full(_lib.PLAN_CANDIDATES, np.nan, dtype=np.float64)
    failed = np.zeros(_lib.PLAN_CANDIDATES, dtype=np.float64)  # time of a run that overflowed
    for c, p in enumerate(cands):
        if p is None:
            continue
        t, st = _time_join(d, p, ws, nb, out)
        if st == _lib.OK:
            times[c] = t
        else:
            failed[c] = t
    t_exact, st = _time_join(d, exact, ws, nb, out)
    check(st, "exact plan")
    times[_lib.PLAN_CANDIDATE_EXACT] = t_exact
    return feat, times, failed, t_exact


def targets(times: np.ndarray, failed: Optional[np.ndarray] = None, t_exact: Optional[np.ndarray] = None):
    """Relative log2 times (minus the workload's mean) and the mask of the
    candidates that carry a target.  A candidate that overflowed on the
    device costs its run plus the exact plan's (what choosing it costs), so
    the network learns to avoid it; candidates that could not be built are
    masked out."""
    if failed is not None and t_exact is not None:
        ran_out = np.isnan(times) & (failed > 0)
        times = np.where(ran_out, failed + t_exact[:, None], times)
    lt = np.log2(np.where(np.isnan(times), 1.0, times))
    mask = (~np.isnan(times)).astype(np.float32)
    mean = (lt * mask).sum(1, keepdims=True) / np.maximum(mask.sum(1, keepdims=True), 1)
    return ((lt - mean) * mask).astype(np.float32), mask


def evaluate(pred: np.ndarray, times: np.ndarray, failed: np.ndarray, t_exact: np.ndarray):
    """Learned choice against the exact plan, per workload: the best-ranked
    candidate that can be built (as pj_plan_learned picks it), its time, or,
    when it overflowed on the device, that run plus the exact plan's (the
    fallback)."""
    buildable = ~np.isnan(times) | (failed > 0)
    choice = np.where(buildable, pred, np.inf).argmin(1)
    rows = np.arange(pred.shape[0])
    t = times[rows, choice]
    fb = np.isnan(t)
    realised = np.where(fb, failed[rows, choice] + t_exact, t)
    speed = t_exact / realised
    best = np.nanmin(times, 1)
    return {"geomean_speedup_vs_exact": float(np.exp(np.log(speed).mean())),
            "mean_speedup_vs_exact": float(speed.mean()),
            "fallback_rate": float(fb.mean()),
            "geomean_oracle_best_vs_exact": float(np.exp(np.log(t_exact / best).mean())),
            "workloads": int(pred.shape[0])}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", action="store_true")
    ap.add_argument("--workloads", type=int, default=400)
    ap.add_argument("--held-out", type=float, default=0.25)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--seed", type=int, default=11)
    ap.add_argument("--min-log2-build", type=int, default=18)
    ap.add_argument("--max-log2-build", type=int, default=28)
    ap.add_argument("--max-log2-probe", type=int, default=29)
    ap.add_argument("--out", default=WEIGHTS)
    ap.add_argument("--data", default="", help="save the sweep (npz) here")
    ap.add_argument("--from-data", default="",
                    help="train on saved sweeps (comma-separated npz files from --data) instead of sweeping")
    a = ap.parse_args()
    rng = np.random.default_rng(a.seed)
    F, T, FAIL, TEX, META = [], [], [], [], []
    t0 = time.time()
    if a.from_data:
        for path in a.from_data.split(","):
            z = np.load(path)
            F += list(z["features"])
            T += list(z["times"])
            FAIL += list(z["failed"])
            TEX += list(z["t_exact"])
            META += json.loads(str(z["meta"]))
        # shuffle with the seed so that the held-out split mixes the sweeps
        order = rng.permutation(len(F))
        F, T, FAIL, TEX, META = ([x[i] for i in order] for x in (F, T, FAIL, TEX, META))
        a.workloads = len(F)
    for i in range(0 if a.from_data else a.workloads):
        b, p, meta = sweep_workload(rng, a.max_log2_build, a.max_log2_probe, min_log2_build=a.min_log2_build)
        f, t, fl, te = measure(b, p)
        F.append(f), T.append(t), FAIL.append(fl), TEX.append(te), META.append(meta)
        del b, p
    F, T, FAIL, TEX = (np.array(x) for x in (F, T, FAIL, TEX))
    if a.data and not a.from_data:
        np.savez(a.data, features=F, times=T, failed=FAIL, t_exact=TEX, meta=json.dumps(META))
    tgt, mask = targets(T, FAIL, TEX)
    n_test = int(round(a.held_out * len(F)))
    tr, te = slice(n_test, None), slice(0, n_test)
    net = Mlp(seed=a.seed)
    losses = net.train(F[tr], tgt[tr], mask[tr], steps=a.steps)
    report = {"train": evaluate(net.predict(F[tr]), T[tr], FAIL[tr], TEX[tr]),
              "held_out": evaluate(net.predict(F[te]), T[te], FAIL[te], TEX[te]),
              "loss_first_last": [losses[0], losses[-1]], "sweep_seconds": time.time() - t0,
              "sweep": {"workloads": a.workloads, "seed": a.seed, "min_log2_build": a.min_log2_build,
                        "max_log2_build": a.max_log2_build, "max_log2_probe": a.max_log2_probe,
                        "from_data": a.from_data},
        "candidates": _lib.PLAN_CANDIDATES}
    np.savez(a.out, params=net.params.cpu().numpy(), report=json.dumps(report))
    print(json.dumps(report))


if __name__ == "__main__":
    main()
