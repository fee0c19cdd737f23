"""The oracle: a CPU restatement of the reference join path, plus loaders for
the reference's own code compiled into oracle/_ref.

TEST INFRASTRUCTURE ONLY -- imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline / reference legs as the checker.  The product path
(partitioned_join_b200) never imports it.
"""
