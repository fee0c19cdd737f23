"""partitioned_join_b200 -- a B200-native (sm_100a) radix-partitioned inner
equi-join behind the C ABI of include/pj.h.

The native library (libpj.so) is built in-tree by
`python -m partitioned_join_b200.build`; importing the package does not
build it, and every operation raises if it is missing.
"""
from ._lib import (DIGIT_HASH, DIGIT_RAW, SLOT_FAST, SLOT_REF, SPLIT_HASH, SPLIT_POSITION, TABLE_BUCKET, TABLE_COMPACT, TABLE_EXACT,
                   TABLE_OPEN, JoinDesc, Output, PJError, Plan)

__all__ = ["DIGIT_HASH", "DIGIT_RAW", "SLOT_FAST", "SLOT_REF", "SPLIT_HASH", "SPLIT_POSITION", "TABLE_BUCKET",
           "TABLE_COMPACT", "TABLE_EXACT", "TABLE_OPEN", "JoinDesc",
           "Output", "PJError", "Plan", "api", "datagen"]


def __getattr__(name):
    if name in ("api", "datagen"):
        import importlib
        return importlib.import_module(f".{name}", __name__)
    if name in ("partitioned_join", "join_count", "plan_default", "plan_exact", "hash_keys", "hash_slots",
                "radix_histogram", "partition", "Joiner"):
        from . import api
        return getattr(api, name)
    raise AttributeError(name)
