"""pj_inner_join_noalloc: the join on the library's built-in workspace.

Collected last on purpose: the built-in workspace is per-process state, and
these tests must pass both alone and after every other test has run joins on
the same device.  Two joins in a row on the built-in workspace must each
give exactly the oracle's pairs (oracle.inner_join, the restatement of the
reference's inner_join_cpu), which are also the pairs pj_inner_join gives
with a caller workspace."""
import ctypes

import numpy as np
import pytest
import torch

from oracle import oracle
from partitioned_join_b200 import _lib, api, datagen
from partitioned_join_b200._lib import PJError


def _sorted(br, pr):
    return oracle.sorted_pairs(br.cpu().numpy(), pr.cpu().numpy())


def test_noalloc_rejects_oversized_join_before_device_work():
    # sizes only: the workspace check runs before the device is touched
    d = api.desc_for_sizes(1 << 24, 1 << 24, 4)
    need = api.workspace_size(d)
    assert need > _lib.NOALLOC_SCRATCH_BYTES
    out = _lib.Output()
    out.build_row, out.probe_row, out.capacity, out.count = 16, 16, 1 << 24, 16
    st = _lib.lib().pj_inner_join_noalloc(ctypes.byref(d), None, ctypes.byref(out), None)
    assert st == _lib.ERR_WORKSPACE


def test_noalloc_rejects_invalid_arguments():
    out = _lib.Output()
    assert _lib.lib().pj_inner_join_noalloc(None, None, ctypes.byref(out), None) == _lib.ERR_INVALID


@pytest.mark.gpu
def test_noalloc_two_calls_match_pj_inner_join():
    dev = "cuda:0"
    cases = [datagen.config2(seed=31, n_build=1 << 20, n_probe=1 << 22),   # near the size limit
             datagen.config1(seed=32, n_build=1 << 16, n_probe=1 << 18)]   # smaller: stale scratch would show
    inputs, expected = [], []
    for b, p in cases:
        bt = torch.from_numpy(b).to(dev)
        pt = torch.from_numpy(p).to(dev)
        assert api.workspace_size(api.make_desc(bt, pt)) <= _lib.NOALLOC_SCRATCH_BYTES
        inputs.append((bt, pt))
        eb, ep = oracle.inner_join(b, p, True)
        exp = oracle.sorted_pairs(eb, ep)
        assert np.array_equal(_sorted(*api.partitioned_join(bt, pt)), exp)
        expected.append(exp)
    # two calls in a row on the built-in workspace
    got = [api.inner_join_noalloc(bt, pt, capacity=pt.numel()) for bt, pt in inputs]
    torch.cuda.synchronize()
    for (gb, gp), exp in zip(got, expected):
        assert np.array_equal(_sorted(gb, gp), exp)


@pytest.mark.gpu
def test_noalloc_oversized_join_rejected_on_device():
    dev = "cuda:0"
    b = torch.arange(1 << 23, dtype=torch.int32, device=dev)
    p = torch.arange(1 << 23, dtype=torch.int32, device=dev)
    with pytest.raises(PJError) as e:
        api.inner_join_noalloc(b, p, capacity=1 << 23)
    assert e.value.status == _lib.ERR_WORKSPACE
