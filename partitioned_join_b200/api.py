"""Host-side interface of the B200 join, over the C ABI (include/pj.h).

Mirrors the reference's entry points for this path (the `partitioned_join`
binary's stage sequence, main.cu:762-892) with device tensors in and out:

    partitioned_join(build_keys, probe_keys, unique_build_keys=...)   main.cu:762-892
    join_count(...)                  output sizing, main.cu:697-704 (the reference runs the CPU join)
    radix_histogram(...)             histogram_pass_one / _two, combined_histogram_pass
    partition(...)                   partition_input_tables_pass_one / _two
    hash_keys(...), hash_slots(...)  MurmurHash3_32 and the table slot of hash_join
    plan_default(...), plan_exact(...)  the -n/-N/-f choice and handle_skewed_data's sizing

Torch provides device memory and streams only; every computation runs in
libpj.so's sm_100a kernels.  Errors raise PJError (the reference prints and
continues, common.cuh:14-20).
"""
from __future__ import annotations

import ctypes
from typing import Optional, Tuple

import torch

from . import _lib
from ._lib import JoinDesc, Output, PJError, Plan, check, lib

KEY_DTYPES = {torch.int32: 4, torch.int64: 8}


def _stream_ptr(stream) -> Optional[int]:
    if stream is None:
        stream = torch.cuda.current_stream()
    return ctypes.c_void_p(stream.cuda_stream)


def _keys(t: torch.Tensor, name: str) -> torch.Tensor:
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError(f"{name} must be a CUDA tensor")
    if t.dtype not in KEY_DTYPES:
        raise TypeError(f"{name} must be int32 or int64")
    if t.dim() != 1:
        raise ValueError(f"{name} must be one-dimensional")
    if not t.is_contiguous():
        t = t.contiguous()
    return t


PAYLOAD_DTYPES = {torch.int32: 4, torch.int64: 8, torch.float32: 4, torch.float64: 8}


def make_desc(build_keys: torch.Tensor, probe_keys: torch.Tensor, unique_build_keys: bool = True,
              build_payload: Optional[torch.Tensor] = None, probe_payload: Optional[torch.Tensor] = None) -> JoinDesc:
    b = _keys(build_keys, "build_keys")
    p = _keys(probe_keys, "probe_keys")
    if b.dtype != p.dtype:
        raise TypeError("build and probe keys must have the same dtype")
    d = JoinDesc()
    d.build_keys = b.data_ptr() if b.numel() else None
    d.probe_keys = p.data_ptr() if p.numel() else None
    d.n_build = b.numel()
    d.n_probe = p.numel()
    d.key_bytes = KEY_DTYPES[b.dtype]
    d.payload_bytes = 0
    d.unique_build_keys = 1 if unique_build_keys else 0
    pays = [(t, n, side) for t, n, side in ((build_payload, b.numel(), "build"), (probe_payload, p.numel(), "probe"))
            if t is not None]
    for t, n, side in pays:
        if not t.is_cuda or t.dim() != 1 or t.numel() != n or t.dtype not in PAYLOAD_DTYPES or not t.is_contiguous():
            raise ValueError(f"{side}_payload must be a contiguous CUDA column of 4- or 8-byte values, one per key")
    if pays:
        widths = {PAYLOAD_DTYPES[t.dtype] for t, _, _ in pays}
        if len(widths) != 1:
            raise ValueError("build and probe payloads must have the same width")
        d.payload_bytes = widths.pop()
        if build_payload is not None:
            d.build_payload = build_payload.data_ptr()
        if probe_payload is not None:
            d.probe_payload = probe_payload.data_ptr()
    return d


def desc_for_sizes(n_build: int, n_probe: int, key_bytes: int = 4, unique_build_keys: bool = True) -> JoinDesc:
    d = JoinDesc()
    d.build_keys = 16 if n_build else None  # planning needs no memory; a non-null marker only
    d.probe_keys = 16 if n_probe else None
    d.n_build, d.n_probe, d.key_bytes = n_build, n_probe, key_bytes
    d.unique_build_keys = 1 if unique_build_keys else 0
    return d


def plan_default(n_build: int, n_probe: int, key_bytes: int = 4, unique_build_keys: bool = True) -> Plan:
    """Plan from sizes alone (pj_plan_default)."""
    p = Plan()
    check(lib().pj_plan_default(ctypes.byref(desc_for_sizes(n_build, n_probe, key_bytes, unique_build_keys)),
                                ctypes.byref(p)), "pj_plan_default")
    return p


def workspace_size(desc: JoinDesc, plan: Optional[Plan] = None) -> int:
    n = ctypes.c_size_t(0)
    check(lib().pj_workspace_size(ctypes.byref(desc), ctypes.byref(plan) if plan is not None else None,
                                  ctypes.byref(n)), "pj_workspace_size")
    return n.value


def alloc_workspace(nbytes: int, device) -> torch.Tensor:
    # torch's caching allocator returns 512-byte aligned blocks
    ws = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=device)
    assert ws.data_ptr() % 256 == 0
    return ws


class Joiner:
    """Reusable join context: workspace and output buffers sized once for a
    (sizes, plan), so repeated joins allocate nothing (bench and batch use)."""

    def __init__(self, build_keys: torch.Tensor, probe_keys: torch.Tensor, unique_build_keys: bool = True,
                 plan: Optional[Plan] = None, capacity: Optional[int] = None, plan_per_call: bool = False):
        """plan_per_call: every launch passes a null plan, so the library
        plans from the sizes (pj_plan_default) inside each call; `plan` must
        then be that same default plan (the workspace is sized for it)."""
        self.plan_per_call = plan_per_call
        self.build_keys = _keys(build_keys, "build_keys")
        self.probe_keys = _keys(probe_keys, "probe_keys")
        self.unique = unique_build_keys
        self.desc = make_desc(self.build_keys, self.probe_keys, unique_build_keys)
        self.plan = plan if plan is not None else plan_default(self.desc.n_build, self.desc.n_probe,
                                                               self.desc.key_bytes, unique_build_keys)
        if plan_per_call:
            default = plan_default(self.desc.n_build, self.desc.n_probe, self.desc.key_bytes, unique_build_keys)
            if default.as_dict() != self.plan.as_dict():
                raise ValueError("plan_per_call needs the size-only default plan")
        dev = self.build_keys.device
        self.ws_bytes = workspace_size(self.desc, self.plan)
        self.ws = alloc_workspace(self.ws_bytes, dev)
        if capacity is None:
            capacity = self.desc.n_probe if unique_build_keys else self._count()
        self.capacity = int(capacity)
        self.build_row = torch.empty(max(self.capacity, 1), dtype=torch.int32, device=dev)
        self.probe_row = torch.empty(max(self.capacity, 1), dtype=torch.int32, device=dev)
        self.count = torch.zeros(1, dtype=torch.int64, device=dev)

    def _count(self) -> int:
        cnt = torch.zeros(1, dtype=torch.int64, device=self.build_keys.device)
        st = _stream_ptr(None)
        check(lib().pj_join_count(ctypes.byref(self.desc), ctypes.byref(self.plan), ctypes.c_void_p(cnt.data_ptr()),
                                  ctypes.c_void_p(self.ws.data_ptr()), self.ws_bytes, st), "pj_join_count")
        check(lib().pj_check(ctypes.c_void_p(self.ws.data_ptr()), st), "pj_join_count")
        return int(cnt.item())

    def launch(self, stream=None) -> None:
        """Enqueue the join on the stream (asynchronous)."""
        check(lib().pj_inner_join(ctypes.byref(self.desc), self._plan_arg(), ctypes.byref(self._out()),
                                  ctypes.c_void_p(self.ws.data_ptr()), self.ws_bytes, _stream_ptr(stream)),
              "pj_inner_join")

    def _plan_arg(self):
        return None if self.plan_per_call else ctypes.byref(self.plan)

    def _out(self) -> Output:
        out = Output()
        out.build_row = self.build_row.data_ptr()
        out.probe_row = self.probe_row.data_ptr()
        out.capacity = self.capacity
        out.count = self.count.data_ptr()
        return out

    def launch_with_events(self, events, stream=None) -> None:
        """Enqueue the join recording one torch.cuda.Event per stage
        (len(events) == len(_lib.STAGES)); the events must already exist
        (recorded once)."""
        arr = (ctypes.c_void_p * len(events))(*[e.cuda_event for e in events])
        check(lib().pj_inner_join_events(ctypes.byref(self.desc), self._plan_arg(), ctypes.byref(self._out()),
                                         ctypes.c_void_p(self.ws.data_ptr()), self.ws_bytes, _stream_ptr(stream), arr),
              "pj_inner_join_events")

    def launch_timed(self, stream=None):
        """Run once with per-stage timers (synchronising); returns {stage: ms}."""
        ms = (ctypes.c_float * len(_lib.STAGES))()
        check(lib().pj_inner_join_timed(ctypes.byref(self.desc), self._plan_arg(), ctypes.byref(self._out()),
                                        ctypes.c_void_p(self.ws.data_ptr()), self.ws_bytes, _stream_ptr(stream), ms),
              "pj_inner_join_timed")
        return dict(zip(_lib.STAGES, list(ms)))

    def status(self, stream=None) -> int:
        """Synchronise and return the device-side status (pj_check)."""
        return lib().pj_check(ctypes.c_void_p(self.ws.data_ptr()), _stream_ptr(stream))

    def result(self, stream=None) -> Tuple[torch.Tensor, torch.Tensor]:
        st = self.status(stream)
        n = int(self.count.item())
        if st == _lib.ERR_CAPACITY:
            raise PJError(st, f"need capacity {n}, have {self.capacity}")
        check(st, "pj_inner_join")
        return self.build_row[:n], self.probe_row[:n]


def partitioned_join(build_keys: torch.Tensor, probe_keys: torch.Tensor, unique_build_keys: bool = True,
                     plan: Optional[Plan] = None, capacity: Optional[int] = None,
                     stream=None) -> Tuple[torch.Tensor, torch.Tensor]:
    """Inner equi-join of two key columns: (build_row, probe_row) int32
    tensors, one entry per matching pair, in no particular order.  The
    reference's stage sequence main.cu:762-892 with its output contract
    (inner_join_cpu.hpp:24-107) carried as row indices."""
    j = Joiner(build_keys, probe_keys, unique_build_keys, plan, capacity)
    j.launch(stream)
    st = j.status(stream)
    if st == _lib.ERR_CAPACITY and capacity is None:
        n = int(j.count.item())
        j = Joiner(build_keys, probe_keys, unique_build_keys, j.plan, n)
        j.launch(stream)
    return j.result(stream)


def partitioned_join_payload(build_keys: torch.Tensor, probe_keys: torch.Tensor,
                             build_payload: Optional[torch.Tensor], probe_payload: Optional[torch.Tensor],
                             unique_build_keys: bool = True, plan: Optional[Plan] = None, stream=None):
    """The join plus payload materialisation: (build_row, probe_row,
    build_payload[build_row], probe_payload[probe_row]) -- the reference's
    joined {key, probe_val} records (hash_join_kernels.cuh:155-163) as
    columns.  A payload argument may be None (its output is then None)."""
    b = _keys(build_keys, "build_keys")
    p = _keys(probe_keys, "probe_keys")
    desc = make_desc(b, p, unique_build_keys, build_payload, probe_payload)
    j = Joiner(b, p, unique_build_keys, plan)  # output sized by pj_join_count for repeated keys
    dev = b.device
    pb = torch.empty(max(j.capacity, 1), dtype=build_payload.dtype, device=dev) if build_payload is not None else None
    pp = torch.empty(max(j.capacity, 1), dtype=probe_payload.dtype, device=dev) if probe_payload is not None else None
    out = j._out()
    out.build_payload_out = pb.data_ptr() if pb is not None else None
    out.probe_payload_out = pp.data_ptr() if pp is not None else None
    check(lib().pj_inner_join(ctypes.byref(desc), ctypes.byref(j.plan), ctypes.byref(out),
                              ctypes.c_void_p(j.ws.data_ptr()), j.ws_bytes, _stream_ptr(stream)), "pj_inner_join")
    check(j.status(stream), "pj_inner_join")
    n = int(j.count.item())
    return (j.build_row[:n], j.probe_row[:n], pb[:n] if pb is not None else None,
            pp[:n] if pp is not None else None)


def generate_tables(n_build: int, n_probe: int, key_dtype=torch.int32, rand_max: Optional[int] = None,
                    selectivity: float = 1.0, unique_build_keys: bool = True, zipf_theta: float = 0.0,
                    seed: int = 1, device="cuda", stream=None):
    """Seeded input tables generated on the device (pj_generate_tables): the
    reference's generate_input_tables recipe plus Zipf-distributed probe
    hits.  rand_max defaults to n_build - 1 (unique keys: a permutation of
    0..n_build-1).  Returns (build_keys, probe_keys, hits), hits = probe rows
    drawn from the build side."""
    kb = KEY_DTYPES[key_dtype]
    if rand_max is None:
        rand_max = max(n_build - 1, 0)
    b = torch.empty(max(n_build, 1), dtype=key_dtype, device=device)[:n_build]
    p = torch.empty(max(n_probe, 1), dtype=key_dtype, device=device)[:n_probe]
    hits = torch.zeros(1, dtype=torch.int64, device=device)
    check(lib().pj_generate_tables(ctypes.c_void_p(b.data_ptr()), n_build, ctypes.c_void_p(p.data_ptr()), n_probe, kb,
                                   rand_max, float(selectivity), 1 if unique_build_keys else 0, float(zipf_theta),
                                   seed & (2**64 - 1), ctypes.c_void_p(hits.data_ptr()), _stream_ptr(stream)),
          "pj_generate_tables")
    return b, p, int(hits.item())


class BatchJoiner:
    """A batch of joins (pj_join_batch): joins whose build side fits one
    shared-memory table run in one persistent launch draining a (join, probe
    chunk) queue; the others take the partitioned path.  Outputs and the
    workspace are allocated once; launch() only enqueues kernels, so it can
    be captured in a CUDA graph (see graph())."""

    def __init__(self, pairs, unique_build_keys: bool = True, config: Optional[_lib.BatchConfig] = None):
        self.pairs = [(_keys(b, "build_keys"), _keys(p, "probe_keys")) for b, p in pairs]
        n = len(self.pairs)
        self.n = n
        dev = self.pairs[0][0].device
        kb = KEY_DTYPES[self.pairs[0][0].dtype]
        self.descs = (JoinDesc * n)(*[make_desc(b, p, unique_build_keys) for b, p in self.pairs])
        self.config = config if config is not None else batch_config_default(kb)
        self.capacity = [int(p.numel()) if unique_build_keys else join_count(b, p, False) for b, p in self.pairs]
        self.build_row = [torch.empty(max(c, 1), dtype=torch.int32, device=dev) for c in self.capacity]
        self.probe_row = [torch.empty(max(c, 1), dtype=torch.int32, device=dev) for c in self.capacity]
        self.count = torch.zeros(n, dtype=torch.int64, device=dev)
        outs = []
        for i in range(n):
            o = Output()
            o.build_row, o.probe_row = self.build_row[i].data_ptr(), self.probe_row[i].data_ptr()
            o.capacity, o.count = self.capacity[i], self.count.data_ptr() + 8 * i
            outs.append(o)
        self.outs = (Output * n)(*outs)
        # room for every configuration the autotuner may try (all joins partitioned)
        worst = _lib.BatchConfig.from_buffer_copy(self.config)
        worst.direct_max_build = 0
        self.ws_bytes = max(self._ws_size(self.config), self._ws_size(worst))
        for together in (1, 0):
            for d in (-1, 0, 1):
                c = _lib.BatchConfig.from_buffer_copy(worst)
                c.large_bits_delta = d
                c.large_batched = together
                try:
                    self.ws_bytes = max(self.ws_bytes, self._ws_size(c))
                except PJError:
                    pass
        self.ws = alloc_workspace(self.ws_bytes, dev)
        self.prepare()

    def _ws_size(self, cfg) -> int:
        nb = ctypes.c_size_t(0)
        check(lib().pj_batch_workspace_size(self.descs, self.n, ctypes.byref(cfg), ctypes.byref(nb)),
              "pj_batch_workspace_size")
        return nb.value

    def prepare(self, stream=None) -> None:
        check(lib().pj_batch_prepare(self.descs, self.outs, self.n, ctypes.byref(self.config),
                                     ctypes.c_void_p(self.ws.data_ptr()), self.ws_bytes, _stream_ptr(stream)),
              "pj_batch_prepare")

    def launch(self, stream=None) -> None:
        check(lib().pj_join_batch(self.descs, self.outs, self.n, ctypes.byref(self.config),
                                  ctypes.c_void_p(self.ws.data_ptr()), self.ws_bytes, _stream_ptr(stream)),
              "pj_join_batch")

    def check(self, stream=None) -> None:
        check(lib().pj_batch_check(ctypes.c_void_p(self.ws.data_ptr()), _stream_ptr(stream)), "pj_join_batch")

    def autotune(self, stream=None) -> float:
        best = _lib.BatchConfig()
        ms = ctypes.c_float(0)
        check(lib().pj_batch_autotune(self.descs, self.outs, self.n, ctypes.c_void_p(self.ws.data_ptr()),
                                      self.ws_bytes, _stream_ptr(stream), ctypes.byref(best), ctypes.byref(ms)),
              "pj_batch_autotune")
        self.config = best
        self.prepare(stream)
        return ms.value

    def graph(self):
        """A CUDA graph of one launch() (replay with .replay())."""
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            self.launch(s)  # warm-up outside capture: kernel attributes, module loads
        torch.cuda.current_stream().wait_stream(s)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.launch()
        return g

    def results(self):
        self.check()
        counts = self.count.cpu().tolist()
        return [(self.build_row[i][: counts[i]], self.probe_row[i][: counts[i]]) for i in range(self.n)]


def batch_config_default(key_bytes: int = 4) -> _lib.BatchConfig:
    c = _lib.BatchConfig()
    check(lib().pj_batch_config_default(key_bytes, ctypes.byref(c)), "pj_batch_config_default")
    return c


def inner_join_noalloc(build_keys: torch.Tensor, probe_keys: torch.Tensor, capacity: int,
                       unique_build_keys: bool = True, plan: Optional[Plan] = None,
                       stream=None) -> Tuple[torch.Tensor, torch.Tensor]:
    """The join through pj_inner_join_noalloc: the library uses its built-in
    64 MiB workspace instead of one allocated here, so only the output
    columns (capacity pairs) are allocated by the caller.  Raises PJError
    (workspace) for joins too large for that workspace.  Synchronises the
    stream."""
    b = _keys(build_keys, "build_keys")
    p = _keys(probe_keys, "probe_keys")
    desc = make_desc(b, p, unique_build_keys)
    dev = b.device
    build_row = torch.empty(max(capacity, 1), dtype=torch.int32, device=dev)
    probe_row = torch.empty(max(capacity, 1), dtype=torch.int32, device=dev)
    count = torch.zeros(1, dtype=torch.int64, device=dev)
    out = Output()
    out.build_row, out.probe_row = build_row.data_ptr(), probe_row.data_ptr()
    out.capacity, out.count = capacity, count.data_ptr()
    check(lib().pj_inner_join_noalloc(ctypes.byref(desc), ctypes.byref(plan) if plan is not None else None,
                                      ctypes.byref(out), _stream_ptr(stream)), "pj_inner_join_noalloc")
    n = int(count.item())
    return build_row[:n], probe_row[:n]


def join_count(build_keys: torch.Tensor, probe_keys: torch.Tensor, unique_build_keys: bool = True,
               plan: Optional[Plan] = None) -> int:
    d = make_desc(build_keys, probe_keys, unique_build_keys)
    if plan is None:
        plan = plan_default(d.n_build, d.n_probe, d.key_bytes, unique_build_keys)
    nb = workspace_size(d, plan)
    ws = alloc_workspace(nb, build_keys.device)
    cnt = torch.zeros(1, dtype=torch.int64, device=build_keys.device)
    st = _stream_ptr(None)
    check(lib().pj_join_count(ctypes.byref(d), ctypes.byref(plan), ctypes.c_void_p(cnt.data_ptr()),
                              ctypes.c_void_p(ws.data_ptr()), nb, st), "pj_join_count")
    check(lib().pj_check(ctypes.c_void_p(ws.data_ptr()), st), "pj_join_count")
    return int(cnt.item())


def plan_exact(build_keys: torch.Tensor, probe_keys: torch.Tensor, unique_build_keys: bool = True,
               ws: Optional[torch.Tensor] = None) -> Plan:
    """The exact-histogram plan (pj_plan_exact).  ws: a workspace of at
    least the default plan's size to reuse (else one is allocated)."""
    d = make_desc(build_keys, probe_keys, unique_build_keys)
    base = plan_default(d.n_build, d.n_probe, d.key_bytes, unique_build_keys)
    nb = workspace_size(d, base)
    if ws is None or ws.numel() < nb:
        ws = alloc_workspace(nb, build_keys.device)
    p = Plan()
    check(lib().pj_plan_exact(ctypes.byref(d), ctypes.c_void_p(ws.data_ptr()), nb, ctypes.byref(p),
                              _stream_ptr(None)), "pj_plan_exact")
    return p


def hash_keys(keys: torch.Tensor) -> torch.Tensor:
    """MurmurHash3_32 (seed 0) of every key, as int32 bit patterns."""
    k = _keys(keys, "keys")
    out = torch.empty(k.numel(), dtype=torch.int32, device=k.device)
    check(lib().pj_hash_keys(ctypes.c_void_p(k.data_ptr()), k.numel(), KEY_DTYPES[k.dtype],
                             ctypes.c_void_p(out.data_ptr()), _stream_ptr(None)), "pj_hash_keys")
    return out


def hash_slots(keys: torch.Tensor, table_slots: int, slot_mode: int = _lib.SLOT_REF, skip_bits: int = 0) -> torch.Tensor:
    k = _keys(keys, "keys")
    out = torch.empty(k.numel(), dtype=torch.int32, device=k.device)
    check(lib().pj_hash_slots(ctypes.c_void_p(k.data_ptr()), k.numel(), KEY_DTYPES[k.dtype], table_slots, slot_mode,
                              skip_bits, ctypes.c_void_p(out.data_ptr()), _stream_ptr(None)), "pj_hash_slots")
    return out


def radix_histogram(keys: torch.Tensor, digit_mode: int, bits1: int, bits2: int = 0, which: int = 0) -> torch.Tensor:
    k = _keys(keys, "keys")
    nb = bits1 if which == 1 else bits2 if which == 2 else bits1 + bits2
    out = torch.empty(1 << nb, dtype=torch.int32, device=k.device)
    check(lib().pj_radix_histogram(ctypes.c_void_p(k.data_ptr()), k.numel(), KEY_DTYPES[k.dtype], digit_mode, bits1,
                                   bits2, which, ctypes.c_void_p(out.data_ptr()), _stream_ptr(None)),
          "pj_radix_histogram")
    return out


def partition(keys: torch.Tensor, plan: Plan) -> Tuple[torch.Tensor, torch.Tensor]:
    """Radix-partition one key column: (tuples as int32 words, offsets[P+1])."""
    k = _keys(keys, "keys")
    kb = KEY_DTYPES[k.dtype]
    cap = ctypes.c_int64(0)
    check(lib().pj_partitioned_capacity(k.numel(), kb, ctypes.byref(plan), ctypes.byref(cap)), "pj_partitioned_capacity")
    words = 2 if kb == 4 else 4
    tuples = torch.empty(cap.value * words + 16, dtype=torch.int32, device=k.device)
    P = 1 << (plan.bits1 + (plan.bits2 if plan.passes == 2 else 0))
    offsets = torch.empty(P + 1, dtype=torch.int64, device=k.device)
    d = desc_for_sizes(k.numel(), 0, kb)
    nb = workspace_size(d, plan)
    ws = alloc_workspace(nb, k.device)
    st = _stream_ptr(None)
    check(lib().pj_partition(ctypes.c_void_p(k.data_ptr()), k.numel(), kb, ctypes.byref(plan),
                             ctypes.c_void_p(tuples.data_ptr()), ctypes.c_void_p(offsets.data_ptr()),
                             ctypes.c_void_p(ws.data_ptr()), nb, st), "pj_partition")
    check(lib().pj_check(ctypes.c_void_p(ws.data_ptr()), st), "pj_partition")
    return tuples, offsets
