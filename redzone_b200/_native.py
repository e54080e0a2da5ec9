"""ctypes binding of ``include/redzone.h`` (``redzone_b200/_lib/libredzone_b200.so``).

There is no fallback: if the native library is absent, importing this module raises.
"""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "_lib" / "libredzone_b200.so"
HEADERS = sorted((PKG.parent / "include").glob("*.h"))

if not LIB_PATH.exists():
    raise ImportError(
        f"redzone_b200 native library not found at {LIB_PATH}; build it with "
        "`python -c 'import __graft_entry__ as g; g.build()'` or `python redzone_b200/build.py`")

lib = ctypes.CDLL(str(LIB_PATH))

c_vp, c_i32, c_u32, c_i64, c_u64, c_f32 = (ctypes.c_void_p, ctypes.c_int32, ctypes.c_uint32,
                                           ctypes.c_int64, ctypes.c_uint64, ctypes.c_float)


RZ_SCHED_AUTO, RZ_SCHED_BLOCK, RZ_SCHED_CLUSTER, RZ_SCHED_GRID, RZ_SCHED_CSCAN, RZ_SCHED_SPLIT, RZ_SCHED_SCANALL = 0, 1, 2, 3, 4, 5, 6


class LaunchCfg(ctypes.Structure):
    _fields_ = [("block", c_i32), ("items", c_i32), ("ctas_per_sm", c_i32), ("use_partition", c_i32),
                ("schedule", c_i32)]

    def as_tuple(self):
        return (self.block, self.items, self.ctas_per_sm, self.use_partition, self.schedule)

    def __repr__(self):
        return (f"LaunchCfg(block={self.block}, items={self.items}, ctas_per_sm={self.ctas_per_sm}, "
                f"partition={self.use_partition}, schedule={self.schedule})")


# Status codes (rz_status).
RZ_OK, RZ_ERR_INVALID_ARG, RZ_ERR_DUPLICATE, RZ_ERR_OUT_OF_RANGE, RZ_ERR_NO_MEMORY, \
    RZ_ERR_TIMEOUT, RZ_ERR_CUDA, RZ_ERR_UNSUPPORTED, RZ_ERR_BUSY = range(9)

# Flags.
RZ_VALIDATE = 0x1
RZ_SYNC = 0x2
RZ_FORCE_PARTITION = 0x4
RZ_FORCE_BLOCK = 0x8
RZ_FORCE_GRID = 0x10
RZ_USE_PREDICTOR = 0x20
RZ_ALLOW_STABLE = 0x40
RZ_CLOBBER_INDICES = 0x80  # accepted; the index list is never written


class ListDesc(ctypes.Structure):
    _fields_ = [("data", c_vp), ("idx", c_vp), ("n", c_i64), ("k", c_i64)]


class BatchCfg(ctypes.Structure):
    _fields_ = [("block", c_i32), ("items", c_i32), ("ctas_per_sm", c_i32), ("span", c_i32), ("wave", c_i32)]

    def as_tuple(self):
        return (self.block, self.items, self.ctas_per_sm, self.span, self.wave)

    def __repr__(self):
        return (f"BatchCfg(block={self.block}, items={self.items}, ctas_per_sm={self.ctas_per_sm}, "
                f"span={self.span}, wave={self.wave})")


class TuneEntry(ctypes.Structure):
    _fields_ = [("cfg", LaunchCfg), ("ms", c_f32)]


class ProducerView(ctypes.Structure):
    _fields_ = [("idx", c_vp), ("counts", c_vp), ("cand", c_vp), ("capacity", c_u32), ("cand_capacity", c_u32),
                ("n", c_u32), ("floor", c_u32)]


def _sig(name, restype, argtypes):
    f = getattr(lib, name)
    f.restype = restype
    f.argtypes = argtypes
    return f


_sig("rz_create", c_i32, [ctypes.POINTER(c_vp), c_i32])
_sig("rz_destroy", None, [c_vp])
_sig("rz_status_string", c_i32, [c_i32, ctypes.c_char_p, ctypes.c_size_t])
_sig("rz_last_cuda_error", c_i32, [c_vp, ctypes.c_char_p, ctypes.c_size_t])
_sig("rz_sync_status", c_i32, [c_vp, c_vp])
_sig("rz_num_sms", c_i32, [c_vp])
_sig("rz_set_scratch_limit", c_i32, [c_vp, c_i64])
_sig("rz_scratch_bytes", c_i64, [c_vp])
_sig("rz_remove", c_i32, [c_vp, c_vp, c_i64, c_u32, c_vp, c_i64, ctypes.POINTER(c_i64), c_u32, c_vp])
_sig("rz_remove_cfg", c_i32, [c_vp, c_vp, c_i64, c_u32, c_vp, c_i64, ctypes.POINTER(LaunchCfg), c_u32, c_vp])
_sig("rz_remove_host_idx", c_i32, [c_vp, c_vp, c_i64, c_u32, c_vp, c_i64, ctypes.POINTER(c_i64), c_u32, c_vp])
_sig("rz_remove_host_idx_async", c_i32, [c_vp, c_vp, c_i64, c_u32, c_vp, c_i64, c_u32, c_vp, ctypes.POINTER(c_u64)])
_sig("rz_wait", c_i32, [c_vp, c_u64, ctypes.POINTER(c_i64)])
_sig("rz_append_remove", c_i32, [c_vp, c_vp, c_i64, c_i64, c_u32, c_vp, c_i64, c_vp, c_i64, ctypes.POINTER(c_i64),
                                  c_u32, c_vp])
_sig("rz_keep", c_i32, [c_vp, c_vp, c_i64, c_u32, c_vp, c_i64, ctypes.POINTER(c_i64), c_u32, c_vp])
_sig("rz_keyindex_create", c_i32, [c_vp, c_i64, ctypes.POINTER(c_vp)])
_sig("rz_keyindex_destroy", None, [c_vp])
_sig("rz_keyindex_build", c_i32, [c_vp, c_vp, c_i64, c_u32, c_vp])
_sig("rz_keyindex_insert", c_i32, [c_vp, c_vp, c_i64, c_i64, c_u32, c_vp])
_sig("rz_keyindex_find", c_i32, [c_vp, c_vp, c_i64, c_vp, c_vp])
_sig("rz_remove_by_key", c_i32, [c_vp, c_vp, c_vp, c_i64, c_u32, c_vp, c_i64, ctypes.POINTER(c_i64), c_u32, c_vp])
_sig("rz_partition", c_i32, [c_vp, c_vp, c_i64, c_u32, c_vp, c_i64, ctypes.POINTER(c_i64), c_u32, c_vp])
_sig("rz_default_cfg", c_i32, [c_vp, c_i64, c_i64, c_u32, ctypes.POINTER(LaunchCfg)])
_sig("rz_test_barrier_timeout", c_i32, [c_vp, c_u32, ctypes.POINTER(c_u32)])
_sig("rz_test_empty_launch", c_i32, [c_vp, c_i32, c_i32, c_i32, c_i32, c_vp])
_sig("rz_test_scatter", c_i32, [c_vp, c_vp, c_i64, c_u32, c_vp, c_i64, c_vp])
_sig("rz_test_thrust_remove", c_i32, [c_vp, c_vp, c_i64, c_vp, c_i64, ctypes.POINTER(c_i64), c_vp])
_sig("rz_last_launch", c_i32, [c_vp, ctypes.POINTER(c_i32), ctypes.POINTER(c_i32), ctypes.POINTER(c_i32)])
_sig("rz_remove_noalloc", c_i32, [c_vp, c_i64, c_u32, c_vp, c_i64, ctypes.POINTER(c_i64), c_vp])
_sig("rz_noalloc_sync_status", c_i32, [c_vp])
_sig("rz_config_space", c_i32, [ctypes.POINTER(LaunchCfg), c_i32])
_sig("rz_producer_create", c_i32, [c_vp, c_i64, c_i64, ctypes.POINTER(c_vp)])
_sig("rz_producer_destroy", None, [c_vp])
_sig("rz_producer_reset", c_i32, [c_vp, c_i64, c_vp])
_sig("rz_producer_get_view", c_i32, [c_vp, ctypes.POINTER(ProducerView)])
_sig("rz_remove_produced", c_i32, [c_vp, c_vp, c_vp, c_u32, ctypes.POINTER(c_i64), c_u32, c_vp])
_sig("rz_produce_where_less", c_i32, [c_vp, c_vp, c_u32, c_vp])
_sig("rz_producer_download", c_i32, [c_vp, c_vp, c_i64, ctypes.POINTER(c_i64), ctypes.POINTER(c_i64), c_vp])
_sig("rz_batch_plan_create", c_i32, [c_vp, ctypes.POINTER(ListDesc), c_i32, c_u32, ctypes.POINTER(BatchCfg),
                                     ctypes.POINTER(c_vp)])
_sig("rz_batch_plan_launch", c_i32, [c_vp, c_vp])
_sig("rz_batch_plan_info", c_i32, [c_vp, ctypes.POINTER(c_i32), ctypes.POINTER(c_i32), ctypes.POINTER(c_i32),
                                   ctypes.POINTER(c_i64), ctypes.POINTER(c_i64)])
_sig("rz_batch_plan_destroy", None, [c_vp])
_sig("rz_remove_batched", c_i32, [c_vp, ctypes.POINTER(ListDesc), c_i32, c_u32, c_u32, c_vp])
_sig("rz_autotune_single", c_i32, [c_vp, c_vp, c_i64, c_u32, c_vp, c_i64, c_i32, ctypes.POINTER(TuneEntry), c_i32,
                                   ctypes.POINTER(c_i32)])
_sig("rz_autotune_batched", c_i32, [c_vp, ctypes.POINTER(ListDesc), c_i32, c_u32, c_i32, ctypes.POINTER(BatchCfg),
                                    ctypes.POINTER(c_f32)])
_sig("rz_tune_table_load", c_i32, [c_vp, ctypes.c_char_p])
_sig("rz_tune_table_save", c_i32, [c_vp, ctypes.c_char_p])
_sig("rz_tune_table_set_single", c_i32, [c_vp, c_u32, c_i32, ctypes.POINTER(LaunchCfg)])
_sig("rz_tune_table_set_batched", c_i32, [c_vp, c_u32, ctypes.POINTER(BatchCfg)])


class ServiceCfg(ctypes.Structure):
    _fields_ = [("shards", c_i32), ("slots", c_i32), ("shard_capacity", c_i64), ("record_bytes", c_u32),
                ("max_batches_per_launch", c_i32), ("index_budget_bytes", c_i64), ("floor_rows", c_i64)]


class ServiceStats(ctypes.Structure):
    _fields_ = [("submitted", c_i64), ("completed", c_i64), ("rejected", c_i64), ("rows_deleted", c_i64),
                ("launches", c_i64), ("refills", c_i64), ("rows_appended", c_i64), ("p50_us", ctypes.c_double),
                ("p99_us", ctypes.c_double), ("mean_us", ctypes.c_double), ("max_us", ctypes.c_double),
                ("mean_batches_per_launch", ctypes.c_double), ("busy_seconds", ctypes.c_double)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


RZ_SUBMIT_BORROW = 0x1
_sig("rz_service_create", c_i32, [c_vp, c_vp, ctypes.POINTER(c_i64), ctypes.POINTER(ServiceCfg), ctypes.POINTER(c_vp)])
_sig("rz_service_submit", c_i32, [c_vp, c_i32, c_vp, c_i64, c_u32, ctypes.POINTER(c_u64)])
_sig("rz_service_drain", c_i32, [c_vp, c_i32])
_sig("rz_service_stats_get", c_i32, [c_vp, ctypes.POINTER(ServiceStats)])
_sig("rz_service_reset_stats", c_i32, [c_vp])
_sig("rz_service_lengths", c_i32, [c_vp, ctypes.POINTER(c_i64), ctypes.POINTER(c_i64)])
_sig("rz_service_destroy", None, [c_vp])
_sig("rz_service_checkpoint", c_i32, [c_vp, ctypes.POINTER(c_i64), ctypes.POINTER(c_i64), c_i32])
_sig("rz_service_restore", c_i32, [c_vp, ctypes.POINTER(c_i64), ctypes.POINTER(c_i64)])
_sig("rz_service_run_poisson", c_i32, [c_vp, ctypes.POINTER(c_vp), ctypes.POINTER(c_i64), c_i32, ctypes.c_double,
                                       ctypes.c_double, c_u64, ctypes.POINTER(ServiceStats)])

_FP = ctypes.POINTER(c_f32)
_sig("rz_mlp_param_count", c_i32, [])
_sig("rz_mlp_create", c_i32, [c_vp, c_u64, ctypes.POINTER(c_vp)])
_sig("rz_mlp_destroy", None, [c_vp])
_sig("rz_mlp_get_params", c_i32, [c_vp, _FP, c_i32])
_sig("rz_mlp_set_params", c_i32, [c_vp, _FP, c_i32])
_sig("rz_mlp_features", c_i32, [c_vp, c_vp, c_i64, c_i64, c_u32, _FP])
_sig("rz_mlp_forward", c_i32, [c_vp, _FP, c_i64, _FP])
_sig("rz_mlp_gradients", c_i32, [c_vp, _FP, _FP, c_i64, _FP, _FP])
_sig("rz_mlp_train", c_i32, [c_vp, _FP, _FP, c_i64, c_i32, c_i32, c_f32, c_u64, _FP])
_sig("rz_set_predictor", c_i32, [c_vp, c_vp])
_sig("rz_predict_cfg", c_i32, [c_vp, c_vp, c_i64, c_i64, c_u32, ctypes.POINTER(LaunchCfg)])
_sig("rz_batch_config_space", c_i32, [ctypes.POINTER(BatchCfg), c_i32])
_sig("rz_batch_features", c_i32, [ctypes.POINTER(ListDesc), c_i32, c_u32, _FP])
_sig("rz_set_batch_predictor", c_i32, [c_vp, c_vp])
_sig("rz_predict_batch_cfg", c_i32, [c_vp, ctypes.POINTER(ListDesc), c_i32, c_u32, ctypes.POINTER(BatchCfg)])
_sig("rz_phase_stamps", c_i32, [c_vp, c_i32])
_sig("rz_read_phase_stamps", c_i32, [c_vp, ctypes.POINTER(c_u64), c_i32, ctypes.POINTER(c_i32)])


def status_string(code: int) -> str:
    buf = ctypes.create_string_buffer(128)
    lib.rz_status_string(code, buf, 128)
    return buf.value.decode()


def declared_symbols() -> list[str]:
    """Every function name declared in include/*.h."""
    names = []
    for h in HEADERS:
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for m in re.finditer(r"\b(rz_[a-z0-9_]+)\s*\(", text):
            if m.group(1) not in names:
                names.append(m.group(1))
    return names
