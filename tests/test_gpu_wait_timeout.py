"""Bounded device waits end with an error status, not a hang.

The decoupled look-back scan waits for its predecessor tiles.  Here one
tile withholds its publish (pj_diag_scan_timeout), so every tile after it
polls a few thousand times, gives up and raises the timeout flag; pj_check
reports PJ_ERR_TIMEOUT, the CUDA context stays usable, and the next join on
the same workspace gives the oracle's pairs."""
import ctypes

import numpy as np
import pytest
import torch

from oracle import oracle
from partitioned_join_b200 import _lib, api, datagen

pytestmark = pytest.mark.gpu


def test_lookback_wait_times_out_and_workspace_recovers():
    b, p = datagen.config2(seed=71, n_build=1 << 22, n_probe=1 << 22)
    bt, pt = torch.from_numpy(b).cuda(), torch.from_numpy(p).cuda()
    j = api.Joiner(bt, pt, True)
    L = _lib.lib()
    # the build side's scan covers P1 x scatter CTAs counters, 4096 a tile
    n_tiles = ((1 << j.plan.bits1) * torch.cuda.get_device_properties(0).multi_processor_count + 4095) // 4096
    assert n_tiles >= 3
    ws = ctypes.c_void_p(j.ws.data_ptr())
    st = L.pj_diag_scan_timeout(ctypes.byref(j.desc), ctypes.byref(j.plan), ws, j.ws_bytes, 1, 2000, None)
    assert st == _lib.OK
    assert L.pj_check(ws, None) == _lib.ERR_TIMEOUT
    assert L.pj_check(ws, None) == _lib.OK  # the flag was cleared
    # a tile index the scan does not have is rejected before any launch
    assert L.pj_diag_scan_timeout(ctypes.byref(j.desc), ctypes.byref(j.plan), ws, j.ws_bytes, n_tiles + 5, 2000,
                                  None) == _lib.ERR_INVALID
    # the next join on the same workspace is clean and correct
    j.launch()
    br, pr = j.result()
    eb, ep = oracle.inner_join(b, p, True)
    assert np.array_equal(oracle.sorted_pairs(br.cpu().numpy(), pr.cpu().numpy()), oracle.sorted_pairs(eb, ep))
