"""The key identities EXACT tables rest on, checked on the CPU with the
oracle's MurmurHash3_x86_32 (pinned to the reference's golden vectors):

* a 4-byte key is a bijection of its hash, so equal hashes mean equal keys;
* for an 8-byte key and a fixed low word, the high word maps to the hash
  bijectively, so (low word, hash) fixes the key.

A map that is not a bijection would show collisions among these samples
(about n^2 / 2^33 expected for n random inputs: hundreds here)."""
import numpy as np

from oracle import oracle


def test_hash_of_4_byte_keys_has_no_collisions():
    rng = np.random.default_rng(61)
    keys = np.unique(rng.integers(-(1 << 31), (1 << 31) - 1, size=1 << 22, dtype=np.int64)).astype(np.int32)
    h = oracle.hash_keys(keys)
    assert np.unique(h).shape[0] == keys.shape[0]


def test_hash_of_8_byte_keys_is_injective_in_the_high_word():
    rng = np.random.default_rng(62)
    his = np.unique(rng.integers(0, 1 << 32, size=1 << 21, dtype=np.int64))
    for lo in (0, 1, 0x9E3779B9, 0xFFFFFFFF):
        keys = ((his << 32) | lo).astype(np.uint64).view(np.int64)
        h = oracle.hash_keys(keys)
        assert np.unique(h).shape[0] == his.shape[0]


def test_low_word_and_hash_separate_8_byte_keys():
    # many keys per low word and per hash: the pair is unique all the same
    rng = np.random.default_rng(63)
    lo = rng.integers(0, 1 << 8, size=1 << 21, dtype=np.int64)          # 256 low words only
    hi = rng.integers(0, 1 << 32, size=1 << 21, dtype=np.int64)
    keys = np.unique(((hi << 32) | lo).astype(np.uint64)).view(np.int64)
    h = oracle.hash_keys(keys).astype(np.uint64)
    pair = (h << np.uint64(32)) | (keys.view(np.uint64) & np.uint64(0xFFFFFFFF))
    assert np.unique(pair).shape[0] == keys.shape[0]
