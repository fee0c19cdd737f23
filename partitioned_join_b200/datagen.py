"""Seeded synthetic inputs with the shapes of the benchmark configurations.

The reference generates its tables on the GPU with cuRAND (seed 1234,
generate_input_tables.cuh:35-226) and has a Zipf generator that samples a
CDF lookup table by binary search over a random alphabet permutation
(generate_zipf_input.cuh:21-134, dead code there).  These generators follow
the same recipes with numpy's PCG64 streams so that every run, here and on
the GPU box, sees identical inputs for a seed.  No public dataset is used:
the reference's TPC-H Q4 path needs .tbl files that are not available.
"""
from __future__ import annotations

import numpy as np


def unique_perm_keys(n: int, rng: np.random.Generator, dtype=np.int32, start: int = 1) -> np.ndarray:
    """A seeded permutation of start..start+n-1 (unique build keys)."""
    return (rng.permutation(n) + start).astype(dtype)


def probe_uniform(build: np.ndarray, n: int, match_rate: float, rng: np.random.Generator,
                  miss_lo: int, miss_hi: int) -> np.ndarray:
    """Probe keys drawn uniformly with replacement from the build keys with
    probability match_rate, else uniformly from [miss_lo, miss_hi) (a range
    disjoint from the build keys) -- the selectivity rule of init_probe_tbl
    (generate_input_tables.cuh:82-116)."""
    hit = build[rng.integers(0, build.shape[0], size=n)]
    if match_rate >= 1.0:
        return hit
    miss = rng.integers(miss_lo, miss_hi, size=n).astype(build.dtype)
    return np.where(rng.random(n) < match_rate, hit, miss).astype(build.dtype)


def zipf_cdf(alphabet: int, theta: float) -> np.ndarray:
    """CDF lookup table of a Zipf(theta) law over ranks 1..alphabet
    (gen_zipf_lut, generate_zipf_input.cuh:50-79)."""
    w = 1.0 / np.power(np.arange(1, alphabet + 1, dtype=np.float64), theta)
    c = np.cumsum(w)
    return c / c[-1]


def zipf_ranks(n: int, alphabet: int, theta: float, rng: np.random.Generator) -> np.ndarray:
    """n Zipf-distributed ranks in [0, alphabet): uniform draws mapped
    through the CDF table by binary search (gen_zipf, :85-134)."""
    if theta == 0.0:
        return rng.integers(0, alphabet, size=n)
    cdf = zipf_cdf(alphabet, theta)
    r = np.minimum(np.searchsorted(cdf, rng.random(n), side="left"), alphabet - 1)
    return r


def config1(seed: int = 1, n_build: int = 1 << 20, n_probe: int = 1 << 22):
    """Plain uniform join: unique int32 build keys (a seeded permutation of
    1..n_build, payload = row id), probe keys uniform with replacement from
    the build keys (100 % match)."""
    rng = np.random.default_rng(seed)
    b = unique_perm_keys(n_build, rng)
    p = probe_uniform(b, n_probe, 1.0, rng, 0, 1)
    return b, p


def config2(seed: int = 2, n_build: int = 1 << 27, n_probe: int = 1 << 27, match_rate: float = 0.9):
    """Large uniform join: build = seeded permutation of 1..n_build (int32),
    probe = 90 % uniform from the build keys, 10 % from outside [1, n_build]."""
    rng = np.random.default_rng(seed)
    b = unique_perm_keys(n_build, rng)
    p = probe_uniform(b, n_probe, match_rate, rng, n_build + 1, 2**31 - 1)
    return b, p


def config3(seed: int = 3, theta: float = 1.0, n_build: int = 1 << 26, n_probe: int = 1 << 28):
    """Skewed int64 join: unique random int64 build keys, probe keys sampled
    from them by a Zipf(theta) law over a seeded rank permutation."""
    rng = np.random.default_rng(seed)
    b = np.unique(rng.integers(-(1 << 62), 1 << 62, size=int(n_build * 1.0001) + 64, dtype=np.int64))
    b = b[rng.permutation(b.shape[0])[:n_build]]
    order = rng.permutation(n_build)          # rank -> build position
    ranks = zipf_ranks(n_probe, n_build, theta, rng)
    p = b[order[ranks]]
    return b, p
