"""C ABI checks that need no GPU: the library loads, exports every function
include/pj.h declares, plans from sizes and rejects bad arguments."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    text = open(os.path.join(ROOT, "include", "pj.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pj_[a-z_0-9]+)\s*\(", text)))


@pytest.fixture(scope="module")
def L():
    from partitioned_join_b200 import _lib
    return _lib.lib()


def test_header_symbols_exported(L):
    names = header_functions()
    assert len(names) >= 12
    for n in names:
        assert hasattr(L, n), f"libpj.so does not export {n}"


def test_binding_covers_header():
    from partitioned_join_b200 import _lib
    assert set(header_functions()) == set(_lib.SIGNATURES)


def test_status_strings(L):
    for s in range(9):
        assert L.pj_status_string(s)
    assert b"sm_100a" in L.pj_version()


def test_plan_default_sizes():
    from partitioned_join_b200 import api
    p = api.plan_default(1 << 27, 1 << 27, 4)
    assert p.passes == 1 and p.table_capacity > 0
    # every partition (at the expected size) fits the tables of its splits
    cap = p.table_capacity
    assert (1 << 27) / (1 << p.bits1) <= cap * 64
    small = api.plan_default(1000, 4000, 4)
    assert small.bits1 == 0


def test_workspace_size_grows_with_input():
    from partitioned_join_b200 import api
    a = api.workspace_size(api.desc_for_sizes(1 << 20, 1 << 22))
    b = api.workspace_size(api.desc_for_sizes(1 << 24, 1 << 24))
    assert 0 < a < b


def test_invalid_arguments_rejected(L):
    from partitioned_join_b200 import _lib, api
    d = api.desc_for_sizes(100, 100, 4)
    d.key_bytes = 3
    p = _lib.Plan()
    assert L.pj_plan_default(ctypes.byref(d), ctypes.byref(p)) == _lib.ERR_INVALID
    d = api.desc_for_sizes(100, 100, 4)
    n = ctypes.c_size_t()
    bad = api.plan_default(100, 100, 4)
    bad.passes = 3
    assert L.pj_workspace_size(ctypes.byref(d), ctypes.byref(bad), ctypes.byref(n)) == _lib.ERR_INVALID
    bad = api.plan_default(100, 100, 4)
    bad.table_capacity = 1 << 30
    assert L.pj_workspace_size(ctypes.byref(d), ctypes.byref(bad), ctypes.byref(n)) == _lib.ERR_INVALID
    # the join refuses a workspace that is missing
    out = _lib.Output()
    out.count = 16
    assert L.pj_inner_join(ctypes.byref(d), None, ctypes.byref(out), None, 0, None) == _lib.ERR_WORKSPACE
    assert L.pj_hash_keys(None, 10, 4, None, None) == _lib.ERR_INVALID


def test_plan_radix_follows_the_reference_flags(L):
    """pj_plan_radix: -n P1 [-R -N P2] -f factor (main.cu:239-251,867)."""
    import math

    from partitioned_join_b200 import _lib, api
    d = api.desc_for_sizes(1 << 24, 1 << 24, 4)
    p = _lib.Plan()
    assert L.pj_plan_radix(ctypes.byref(d), 256, 512, ctypes.c_float(3.0), ctypes.byref(p)) == _lib.OK
    assert (p.passes, p.bits1, p.bits2) == (2, 8, 9)
    assert p.digit_mode == _lib.DIGIT_RAW and p.split_mode == _lib.SPLIT_POSITION
    assert p.table_capacity == max(64, math.ceil(3.0 * (1 << 24) / (256 * 512)))
    assert L.pj_plan_radix(ctypes.byref(d), 1024, 0, ctypes.c_float(1.0), ctypes.byref(p)) == _lib.OK
    assert (p.passes, p.bits1, p.bits2) == (1, 10, 0)
    # a build chunk larger than one table is capped at the table
    assert p.table_capacity == api.plan_default(1 << 24, 1 << 24, 4).table_capacity or p.table_capacity < (1 << 24) // 1024 + 1
    n = ctypes.c_size_t()
    assert L.pj_workspace_size(ctypes.byref(d), ctypes.byref(p), ctypes.byref(n)) == _lib.OK
    for bad in ((100, 0, 3.0), (256, 100, 3.0), (256, 0, 0.0), (0, 0, 3.0)):
        assert L.pj_plan_radix(ctypes.byref(d), bad[0], bad[1], ctypes.c_float(bad[2]), ctypes.byref(p)) == \
            _lib.ERR_INVALID, bad


def test_plan_candidates_cover_the_schedule_space(L):
    """pj_plan_candidate: one pass with BUCKET/COMPACT/EXACT tables x radix
    width -1/0/+1 x heavy set (none/all/16 most frequent), two passes, and
    the exact planner's plan (made on the device, so not built here)."""
    from partitioned_join_b200 import _lib, api
    d = api.desc_for_sizes(1 << 24, 1 << 24, 4)
    heavy = _lib.Plan()
    heavy.set_heavy(range(100, 140))
    modes = {}
    for c in range(_lib.PLAN_CANDIDATES):
        p = _lib.Plan()
        st = L.pj_plan_candidate(ctypes.byref(d), c, ctypes.byref(heavy), ctypes.byref(p))
        if c == _lib.PLAN_CANDIDATE_EXACT:
            assert st == _lib.ERR_INVALID
            continue
        if st != _lib.OK:
            continue
        modes[c] = (p.passes, p.table_mode, p.bits1, p.n_heavy)
    assert any(m[1] == _lib.TABLE_BUCKET for m in modes.values())
    assert any(m[1] == _lib.TABLE_COMPACT for m in modes.values())
    assert any(m[1] == _lib.TABLE_EXACT for m in modes.values())
    assert any(m[0] == 2 for m in modes.values())
    assert {m[3] for m in modes.values()} >= {0, 16, 40}
    # the three radix widths of one layout differ by one bit each
    assert modes[0][2] + 1 == modes[3][2] and modes[3][2] + 1 == modes[6][2]
