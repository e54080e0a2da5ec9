"""redzone_b200 -- B200-native Redzone O(k) in-place stream compaction.

Python host mirror of the library's C-ABI (``include/redzone.h``). Arrays are torch CUDA
tensors used as plain device buffers: the first axis enumerates items, the remaining axes form
one item (4, 8, 16 or 32 bytes). Removal indices are int32/uint32 tensors of distinct
positions.

The reference's calls are ``RemoveFromList_GPUWide(List, Length, Removals, RemoveCount,
BlockStore)`` (redzone.hxx:626) and ``redzone_CPU(list, listsize, removals, removecount,
times)`` (Redzone_CPU.hxx:150); ``RemoveFromList`` below keeps that argument order and meaning
and returns the new length instead of leaving it implicit. Unlike the reference it never writes
the removal list, and it reports errors as ``RedzoneError`` instead of exiting.
"""
from __future__ import annotations

import ctypes

from . import _native
from ._native import (LaunchCfg, RZ_ALLOW_STABLE, RZ_CLOBBER_INDICES, RZ_FORCE_BLOCK, RZ_FORCE_GRID,
                      RZ_FORCE_PARTITION, RZ_SYNC, RZ_USE_PREDICTOR, RZ_VALIDATE, status_string)

__all__ = ["Context", "RedzoneError", "LaunchCfg", "RemoveFromList", "remove", "default_context",
           "RZ_VALIDATE", "RZ_SYNC", "RZ_FORCE_PARTITION", "RZ_FORCE_BLOCK", "RZ_FORCE_GRID",
           "RZ_USE_PREDICTOR", "RZ_ALLOW_STABLE", "RZ_CLOBBER_INDICES", "item_bytes"]


class RedzoneError(RuntimeError):
    def __init__(self, code: int, detail: str = ""):
        self.code = code
        msg = f"redzone: {status_string(code)} (status {code})"
        if detail:
            msg += f": {detail}"
        super().__init__(msg)


def item_bytes(t) -> int:
    """Bytes per item of a tensor whose first axis enumerates items."""
    per = t.element_size()
    for s in t.shape[1:]:
        per *= int(s)
    return per


def _stream_handle(stream) -> int | None:
    import torch
    if stream is None:
        # torch's current stream of the current device, as a raw handle (cheaper than building a
        # torch.cuda.Stream object on every call)
        raw = getattr(torch._C, "_cuda_getCurrentRawStream", None)
        if raw is not None:
            return raw(torch.cuda.current_device())
        stream = torch.cuda.current_stream()
    return stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)


class Context:
    """Owns library scratch (bitmap, orphan lists, barrier state) on one device."""

    def __init__(self, device: int = 0):
        h = ctypes.c_void_p()
        st = _native.lib.rz_create(ctypes.byref(h), device)
        if st != 0:
            raise RedzoneError(st, "rz_create")
        self.handle = h
        self.device = device

    def close(self):
        if getattr(self, "handle", None):
            _native.lib.rz_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int, what: str):
        if st != 0:
            buf = ctypes.create_string_buffer(512)
            _native.lib.rz_last_cuda_error(self.handle, buf, 512)
            raise RedzoneError(st, f"{what} {buf.value.decode()}".strip())

    @property
    def num_sms(self) -> int:
        return _native.lib.rz_num_sms(self.handle)

    def set_scratch_limit(self, nbytes: int | None) -> None:
        """Cap the scratch this context may grow (None: no cap)."""
        self._check(_native.lib.rz_set_scratch_limit(self.handle, -1 if nbytes is None else int(nbytes)),
                    "rz_set_scratch_limit")

    @property
    def scratch_bytes(self) -> int:
        return int(_native.lib.rz_scratch_bytes(self.handle))

    def remove(self, data, idx, flags: int = 0, stream=None) -> int:
        """In-place Redzone removal; returns the new length (n - k)."""
        n, k = int(data.shape[0]), int(idx.numel())
        out = ctypes.c_int64(0)
        st = _native.lib.rz_remove(self.handle, ctypes.c_void_p(data.data_ptr()), n, item_bytes(data),
                                   ctypes.c_void_p(idx.data_ptr()), k, ctypes.byref(out), flags,
                                   ctypes.c_void_p(_stream_handle(stream)))
        self._check(st, "rz_remove")
        return out.value

    def remove_cfg(self, data, idx, cfg: LaunchCfg, flags: int = 0, stream=None) -> None:
        n, k = int(data.shape[0]), int(idx.numel())
        st = _native.lib.rz_remove_cfg(self.handle, ctypes.c_void_p(data.data_ptr()), n, item_bytes(data),
                                       ctypes.c_void_p(idx.data_ptr()), k, ctypes.byref(cfg), flags,
                                       ctypes.c_void_p(_stream_handle(stream)))
        self._check(st, "rz_remove_cfg")

    def append_remove(self, data, n: int, gain, idx, flags: int = 0, stream=None) -> int:
        """Append `gain` (device tensor of items) at rows [n, n + g) of `data` (capacity =
        data.shape[0]), then remove rows `idx` from the grown list; returns n + g - k."""
        g, k = int(gain.shape[0]), int(idx.numel())
        out = ctypes.c_int64(0)
        st = _native.lib.rz_append_remove(self.handle, ctypes.c_void_p(data.data_ptr()), n, int(data.shape[0]),
                                          item_bytes(data), ctypes.c_void_p(gain.data_ptr()), g,
                                          ctypes.c_void_p(idx.data_ptr()), k, ctypes.byref(out), flags,
                                          ctypes.c_void_p(_stream_handle(stream)))
        self._check(st, "rz_append_remove")
        return out.value

    def keep(self, data, keep, flags: int = 0, stream=None) -> int:
        """Preserve-list compaction: data[0..m) = (old) data[keep[j]], O(m); returns m."""
        n, m = int(data.shape[0]), int(keep.numel())
        out = ctypes.c_int64(0)
        st = _native.lib.rz_keep(self.handle, ctypes.c_void_p(data.data_ptr()), n, item_bytes(data),
                                 ctypes.c_void_p(keep.data_ptr()), m, ctypes.byref(out), flags,
                                 ctypes.c_void_p(_stream_handle(stream)))
        self._check(st, "rz_keep")
        return out.value

    def partition(self, data, idx, flags: int = 0, stream=None) -> int:
        """O(n) stable partition comparator (survivors keep their order)."""
        n, k = int(data.shape[0]), int(idx.numel())
        out = ctypes.c_int64(0)
        st = _native.lib.rz_partition(self.handle, ctypes.c_void_p(data.data_ptr()), n, item_bytes(data),
                                      ctypes.c_void_p(idx.data_ptr()), k, ctypes.byref(out), flags,
                                      ctypes.c_void_p(_stream_handle(stream)))
        self._check(st, "rz_partition")
        return out.value

    def remove_host_idx(self, data, h_idx, flags: int = 0, stream=None) -> int:
        """Indices in host memory (numpy or pinned torch CPU tensor); synchronous; returns new length."""
        n = int(data.shape[0])
        if hasattr(h_idx, "data_ptr"):
            ptr, k = h_idx.data_ptr(), int(h_idx.numel())
        else:
            ptr, k = h_idx.ctypes.data, int(h_idx.size)
        out = ctypes.c_int64(0)
        st = _native.lib.rz_remove_host_idx(self.handle, ctypes.c_void_p(data.data_ptr()), n, item_bytes(data),
                                            ctypes.c_void_p(ptr), k, ctypes.byref(out), flags,
                                            ctypes.c_void_p(_stream_handle(stream)))
        self._check(st, "rz_remove_host_idx")
        return out.value

    def remove_host_idx_async(self, data, h_idx, flags: int = 0, stream=None) -> int:
        """Pipelined host-index removal (rz_remove_host_idx_async): returns a ticket at once;
        collect the result with ``wait(ticket)``. ``h_idx`` must stay unchanged until then."""
        n = data.shape[0]
        if hasattr(h_idx, "data_ptr"):
            ptr, k = h_idx.data_ptr(), h_idx.numel()
        else:
            ptr, k = h_idx.ctypes.data, h_idx.size
        t = ctypes.c_uint64(0)
        st = _native.lib.rz_remove_host_idx_async(self.handle, data.data_ptr(), n, item_bytes(data), ptr, k, flags,
                                                  _stream_handle(stream), ctypes.byref(t))
        self._check(st, "rz_remove_host_idx_async")
        return t.value

    def wait(self, ticket: int) -> int:
        """Wait for an rz_remove_host_idx_async call; returns its new length or raises."""
        out = ctypes.c_int64(0)
        self._check(_native.lib.rz_wait(self.handle, ctypes.c_uint64(ticket), ctypes.byref(out)), "rz_wait")
        return out.value

    def empty_launch(self, grid: int, block: int, cluster: int = 1, smem: int = 0, stream=None) -> None:
        """Launch an empty kernel of the given shape (the event-timing floor of such a launch)."""
        self._check(_native.lib.rz_test_empty_launch(self.handle, grid, block, cluster, smem,
                                                     ctypes.c_void_p(_stream_handle(stream))), "rz_test_empty_launch")

    def thrust_remove(self, data, idx, stream=None) -> int:
        """The reference's O(n) GPU comparator (mark with -1, then thrust::remove) on an int32
        list; returns the new length."""
        out = ctypes.c_int64(0)
        self._check(_native.lib.rz_test_thrust_remove(self.handle, ctypes.c_void_p(data.data_ptr()), int(data.shape[0]),
                                                      ctypes.c_void_p(idx.data_ptr()), int(idx.numel()),
                                                      ctypes.byref(out), ctypes.c_void_p(_stream_handle(stream))),
                    "rz_test_thrust_remove")
        return out.value

    def scatter(self, data, pos, stream=None) -> None:
        """Plain scattered stores data[pos[i]] = item i (rz_test_scatter): the hole writes alone."""
        self._check(_native.lib.rz_test_scatter(self.handle, ctypes.c_void_p(data.data_ptr()), int(data.shape[0]),
                                                item_bytes(data), ctypes.c_void_p(pos.data_ptr()), int(pos.numel()),
                                                ctypes.c_void_p(_stream_handle(stream))), "rz_test_scatter")

    def sync_status(self, stream=None) -> int:
        return _native.lib.rz_sync_status(self.handle, ctypes.c_void_p(_stream_handle(stream)))

    def default_cfg(self, n: int, k: int, w: int) -> LaunchCfg:
        cfg = LaunchCfg()
        self._check(_native.lib.rz_default_cfg(self.handle, n, k, w, ctypes.byref(cfg)), "rz_default_cfg")
        return cfg

    def last_launch(self) -> tuple[int, int, int]:
        """(kernels launched, grid, block) of the most recent removal call on this context."""
        a, b, c = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        _native.lib.rz_last_launch(self.handle, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
        return a.value, b.value, c.value

    def phase_stamps(self, enable: bool) -> None:
        """Turn per-CTA %globaltimer phase stamps of the Redzone kernels on or off."""
        self._check(_native.lib.rz_phase_stamps(self.handle, 1 if enable else 0), "rz_phase_stamps")

    def read_phase_stamps(self):
        """Stamps of the most recent call as a (ctas, 8) uint64 numpy array (ns)."""
        import numpy as np
        buf = (ctypes.c_uint64 * (1024 * 8))()
        n = ctypes.c_int32(0)
        self._check(_native.lib.rz_read_phase_stamps(self.handle, buf, 1024, ctypes.byref(n)), "rz_read_phase_stamps")
        return np.ctypeslib.as_array(buf)[: n.value * 8].reshape(n.value, 8).copy()

    def test_barrier_timeout(self, spin_limit: int) -> int:
        bits = ctypes.c_uint32(0)
        self._check(_native.lib.rz_test_barrier_timeout(self.handle, spin_limit, ctypes.byref(bits)),
                    "rz_test_barrier_timeout")
        return bits.value


def list_descs(lists) -> "ctypes.Array":
    """[(data_tensor, idx_tensor), ...] -> rz_list_desc array (tensors must stay alive)."""
    arr = (_native.ListDesc * len(lists))()
    for q, (d, i) in enumerate(lists):
        arr[q].data = d.data_ptr() if d.numel() else None
        arr[q].idx = i.data_ptr() if i.numel() else None
        arr[q].n = int(d.shape[0])
        arr[q].k = int(i.numel())
    return arr


class BatchPlan:
    """Many lists removed by one persistent launch, replayed from a CUDA graph (rz_batch_plan_*).

    ``lists`` is a sequence of (data, idx) tensor pairs of the same item width; the tensors must
    stay alive (and in place) as long as the plan is used.
    """

    def __init__(self, ctx: Context, lists, cfg: "_native.BatchCfg | None" = None):
        self.ctx = ctx
        self._descs = list_descs(lists)
        w = item_bytes(lists[0][0]) if lists else 4
        h = ctypes.c_void_p()
        st = _native.lib.rz_batch_plan_create(ctx.handle, self._descs, len(lists), w,
                                              ctypes.byref(cfg) if cfg is not None else None, ctypes.byref(h))
        ctx._check(st, "rz_batch_plan_create")
        self.handle = h

    def launch(self, stream=None) -> None:
        self.ctx._check(_native.lib.rz_batch_plan_launch(self.handle, ctypes.c_void_p(_stream_handle(stream))),
                        "rz_batch_plan_launch")

    def info(self) -> dict:
        g, b, i = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        wi, tk = ctypes.c_int64(), ctypes.c_int64()
        _native.lib.rz_batch_plan_info(self.handle, ctypes.byref(g), ctypes.byref(b), ctypes.byref(i),
                                       ctypes.byref(wi), ctypes.byref(tk))
        return {"grid": g.value, "block": b.value, "items": i.value, "work_items": wi.value, "total_k": tk.value}

    def close(self):
        if getattr(self, "handle", None):
            _native.lib.rz_batch_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def remove_batched(ctx: Context, lists, stream=None) -> None:
    """One-shot batched removal (plan, run, synchronise)."""
    descs = list_descs(lists)
    w = item_bytes(lists[0][0]) if lists else 4
    ctx._check(_native.lib.rz_remove_batched(ctx.handle, descs, len(lists), w, 0,
                                             ctypes.c_void_p(_stream_handle(stream))), "rz_remove_batched")


class KeyIndex:
    """Key -> row index of a table whose records begin with a uint64 key (rz_keyindex_*), kept
    exact by `remove_by_key`."""

    def __init__(self, ctx: Context, capacity: int):
        self.ctx = ctx
        h = ctypes.c_void_p()
        ctx._check(_native.lib.rz_keyindex_create(ctx.handle, int(capacity), ctypes.byref(h)), "rz_keyindex_create")
        self.handle = h

    def build(self, table, n: int | None = None, stream=None) -> None:
        n = int(table.shape[0]) if n is None else int(n)
        self.ctx._check(_native.lib.rz_keyindex_build(self.handle, ctypes.c_void_p(table.data_ptr()), n,
                                                      item_bytes(table), ctypes.c_void_p(_stream_handle(stream))),
                        "rz_keyindex_build")

    def insert(self, table, first: int, count: int, stream=None) -> None:
        self.ctx._check(_native.lib.rz_keyindex_insert(self.handle, ctypes.c_void_p(table.data_ptr()), int(first),
                                                       int(count), item_bytes(table),
                                                       ctypes.c_void_p(_stream_handle(stream))), "rz_keyindex_insert")

    def find(self, keys, stream=None):
        """Rows (int64 tensor, -1 when absent) of a CUDA int64 tensor of keys."""
        import torch
        rows = torch.empty(keys.numel(), dtype=torch.int32, device=keys.device)
        self.ctx._check(_native.lib.rz_keyindex_find(self.handle, ctypes.c_void_p(keys.data_ptr()), keys.numel(),
                                                     ctypes.c_void_p(rows.data_ptr()),
                                                     ctypes.c_void_p(_stream_handle(stream))), "rz_keyindex_find")
        r = rows.to(torch.int64) & 0xFFFFFFFF
        r[r == 0xFFFFFFFF] = -1
        return r

    def remove_by_key(self, table, n: int, keys, flags: int = 0, stream=None) -> int:
        out = ctypes.c_int64(0)
        self.ctx._check(_native.lib.rz_remove_by_key(self.ctx.handle, self.handle, ctypes.c_void_p(table.data_ptr()),
                                                     int(n), item_bytes(table), ctypes.c_void_p(keys.data_ptr()),
                                                     keys.numel(), ctypes.byref(out), flags,
                                                     ctypes.c_void_p(_stream_handle(stream))), "rz_remove_by_key")
        return out.value

    def close(self):
        if getattr(self, "handle", None):
            _native.lib.rz_keyindex_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Producer:
    """A removal list made on the GPU with the red-zone marking fused into its producer
    (rz_producer_*; the device side is rz_emit in include/redzone_device.cuh)."""

    def __init__(self, ctx: Context, capacity: int, cand_capacity: int = 4096):
        self.ctx = ctx
        h = ctypes.c_void_p()
        ctx._check(_native.lib.rz_producer_create(ctx.handle, int(capacity), int(cand_capacity), ctypes.byref(h)),
                   "rz_producer_create")
        self.handle = h

    def reset(self, n: int, stream=None) -> None:
        """Start a round for a list of n rows (zeroes the counts on the stream)."""
        self.ctx._check(_native.lib.rz_producer_reset(self.handle, int(n), ctypes.c_void_p(_stream_handle(stream))),
                        "rz_producer_reset")

    def view(self):
        v = _native.ProducerView()
        self.ctx._check(_native.lib.rz_producer_get_view(self.handle, ctypes.byref(v)), "rz_producer_get_view")
        return v

    def produce_where_less(self, keys, threshold: int, stream=None) -> None:
        """Emit every row i with keys[i] < threshold (keys: CUDA uint32/int32 tensor of n entries)."""
        self.ctx._check(_native.lib.rz_produce_where_less(self.handle, ctypes.c_void_p(keys.data_ptr()),
                                                          int(threshold), ctypes.c_void_p(_stream_handle(stream))),
                        "rz_produce_where_less")

    def download(self, stream=None):
        """(list as a numpy uint32 array, k, candidates emitted); synchronous."""
        import numpy as np
        v = self.view()
        buf = np.zeros(max(1, v.capacity), np.uint32)
        k, c = ctypes.c_int64(0), ctypes.c_int64(0)
        self.ctx._check(_native.lib.rz_producer_download(self.handle, buf.ctypes.data, buf.size, ctypes.byref(k),
                                                         ctypes.byref(c), ctypes.c_void_p(_stream_handle(stream))),
                        "rz_producer_download")
        return buf[: min(k.value, v.capacity)].copy(), k.value, c.value

    def remove(self, data, flags: int = 0, stream=None) -> int:
        """Remove the emitted rows from data[0..n); returns n - k with RZ_SYNC, else -1."""
        out = ctypes.c_int64(0)
        self.ctx._check(_native.lib.rz_remove_produced(self.ctx.handle, self.handle, ctypes.c_void_p(data.data_ptr()),
                                                       item_bytes(data), ctypes.byref(out), flags,
                                                       ctypes.c_void_p(_stream_handle(stream))), "rz_remove_produced")
        return out.value

    def close(self):
        if getattr(self, "handle", None):
            _native.lib.rz_producer_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Service:
    """Streaming delete service over a device-resident table (rz_service_*).

    ``table`` is a CUDA tensor of shards * shard_capacity records (first axis = records); it must
    stay alive while the service runs.
    """

    def __init__(self, ctx: Context, table, shards: int, shard_capacity: int, slots: int = 4,
                 max_batches_per_launch: int = 32, index_budget_bytes: int = 64 << 20, floor_rows: int = 0,
                 initial_len=None):
        self.ctx = ctx
        self.table = table
        cfg = _native.ServiceCfg(shards, slots, shard_capacity, item_bytes(table), max_batches_per_launch,
                                 index_budget_bytes, floor_rows)
        init = None
        if initial_len is not None:
            init = (ctypes.c_int64 * shards)(*[int(x) for x in initial_len])
        h = ctypes.c_void_p()
        ctx._check(_native.lib.rz_service_create(ctx.handle, ctypes.c_void_p(table.data_ptr()), init,
                                                 ctypes.byref(cfg), ctypes.byref(h)), "rz_service_create")
        self.handle = h
        self.shards = shards
        self._lent = []

    def submit(self, shard: int, idx, borrow: bool = False) -> int:
        """Queue a delete batch (numpy uint32/int32 array or pinned CPU tensor); returns its ticket."""
        if hasattr(idx, "data_ptr"):
            ptr, cnt = idx.data_ptr(), int(idx.numel())
        else:
            ptr, cnt = idx.ctypes.data, int(idx.size)
        t = ctypes.c_uint64(0)
        st = _native.lib.rz_service_submit(self.handle, shard, ctypes.c_void_p(ptr), cnt,
                                           _native.RZ_SUBMIT_BORROW if borrow else 0, ctypes.byref(t))
        if borrow:
            self._lent.append(idx)
        if st != 0:
            raise RedzoneError(st, "rz_service_submit")
        return t.value

    def drain(self, timeout_ms: int = 600000) -> None:
        self.ctx._check(_native.lib.rz_service_drain(self.handle, timeout_ms), "rz_service_drain")
        self._lent.clear()

    def stats(self) -> dict:
        s = _native.ServiceStats()
        _native.lib.rz_service_stats_get(self.handle, ctypes.byref(s))
        return s.as_dict()

    def reset_stats(self) -> None:
        _native.lib.rz_service_reset_stats(self.handle)

    def lengths(self) -> tuple[list[int], list[int]]:
        """(host view, device-tracked) live lengths per shard."""
        h = (ctypes.c_int64 * self.shards)()
        d = (ctypes.c_int64 * self.shards)()
        self.ctx._check(_native.lib.rz_service_lengths(self.handle, h, d), "rz_service_lengths")
        return list(h), list(d)

    def checkpoint(self, timeout_ms: int = 600000) -> tuple[list[int], list[int]]:
        """Drain, then (live lengths, refill-appended counts) per shard."""
        ln = (ctypes.c_int64 * self.shards)()
        ap = (ctypes.c_int64 * self.shards)()
        self.ctx._check(_native.lib.rz_service_checkpoint(self.handle, ln, ap, timeout_ms), "rz_service_checkpoint")
        return list(ln), list(ap)

    def restore(self, lengths, appended) -> None:
        ln = (ctypes.c_int64 * self.shards)(*[int(x) for x in lengths])
        ap = (ctypes.c_int64 * self.shards)(*[int(x) for x in appended])
        self.ctx._check(_native.lib.rz_service_restore(self.handle, ln, ap), "rz_service_restore")

    def run_poisson(self, pool, rate: float, seconds: float, seed: int = 0) -> dict:
        """Poisson arrivals of random pool batches (pinned CPU tensors) to random shards."""
        ptrs = (ctypes.c_void_p * len(pool))(*[p.data_ptr() for p in pool])
        cnts = (ctypes.c_int64 * len(pool))(*[int(p.numel()) for p in pool])
        s = _native.ServiceStats()
        self.ctx._check(_native.lib.rz_service_run_poisson(self.handle, ptrs, cnts, len(pool), rate, seconds, seed,
                                                           ctypes.byref(s)), "rz_service_run_poisson")
        return s.as_dict()

    def close(self):
        if getattr(self, "handle", None):
            _native.lib.rz_service_destroy(self.handle)
            self.handle = None
            self._lent.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default: dict[int, Context] = {}


def default_context(device: int | None = None) -> Context:
    import torch
    d = torch.cuda.current_device() if device is None else device
    if d not in _default:
        _default[d] = Context(d)
    return _default[d]


def remove(data, idx, flags: int = 0, stream=None) -> int:
    """Remove the items at positions ``idx`` from ``data`` in place; returns the new length."""
    return default_context(data.device.index).remove(data, idx, flags, stream)


def RemoveFromList(List, Length: int, Removals, RemoveCount: int, flags: int = 0, stream=None) -> int:
    """Reference-shaped call: RemoveFromList_GPUWide(List, Length, Removals, RemoveCount, ...).

    ``List`` must hold at least ``Length`` items and ``Removals`` at least ``RemoveCount`` indices;
    only those prefixes are used. Returns ``Length - RemoveCount``.
    """
    if RemoveCount > Length or Length > List.shape[0] or RemoveCount > Removals.numel():
        raise RedzoneError(_native.RZ_ERR_INVALID_ARG, "RemoveFromList sizes")
    return remove(List[:Length], Removals.reshape(-1)[:RemoveCount], flags, stream)
