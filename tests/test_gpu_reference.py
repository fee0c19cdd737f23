"""Parity with the reference's own GPU path (main.cu:762-892), compiled
unchanged for sm_100a into oracle/_ref by oracle/build_ref.sh.

The reference emits {key, probe_payload} records; with -V semantics and the
probe payload set to the probe row id they form a (key, probe_row) multiset.
Ours is projected through build_row -> build_keys[build_row]; with unique
build keys the projection is injective, so equal multisets are full parity.
Skipped where the reference libraries were not built."""
import numpy as np
import pytest
import torch

from oracle import oracle
from partitioned_join_b200 import api, datagen

pytestmark = pytest.mark.gpu


def _key_probe_multiset(keys, rows):
    return np.sort(keys.astype(np.int64) * (1 << 32) + rows.astype(np.int64))


@pytest.mark.parametrize("key_bytes,log2n,p1,p2,factor", [(4, 22, 256, 512, 3.0), (8, 20, 128, 256, 3.0)])
def test_reference_gpu_path_equals_ours(key_bytes, log2n, p1, p2, factor):
    if not oracle.ref_gpu_available(key_bytes):
        pytest.skip("reference GPU library not built (oracle/build_ref.sh)")
    n = 1 << log2n
    b, p = datagen.config2(seed=41, n_build=n, n_probe=n)
    if key_bytes == 8:
        b = b.astype(np.int64) * 1000003 + (1 << 40)
        p = p.astype(np.int64) * 1000003 + (1 << 40)
    rk, rp, _ = oracle.ref_gpu_partitioned_join(b, p, True, True, True, p1, p2, factor, False)
    br, pr = api.partitioned_join(torch.from_numpy(b).cuda(), torch.from_numpy(p).cuda())
    br, pr = br.cpu().numpy(), pr.cpu().numpy()
    ours = _key_probe_multiset(b[br], pr)
    ref = _key_probe_multiset(rk, rp)
    assert ours.shape == ref.shape and np.array_equal(ours, ref)
    # and both equal the CPU oracle
    eb, ep = oracle.inner_join(b, p, True)
    assert np.array_equal(ours, _key_probe_multiset(b[eb], ep))
