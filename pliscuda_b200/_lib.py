"""ctypes binding of libplis.so (include/plis.h).  Importing this module loads the in-tree library
and raises immediately if it is missing: there is no Python fallback for the step."""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libplis.so")

u32 = ctypes.c_uint32
i32 = ctypes.c_int32
u64 = ctypes.c_uint64
i64 = ctypes.c_int64
f64 = ctypes.c_double
vp = ctypes.c_void_p

PLIS_OK = 0
STATUS_NAMES = {
    0: "PLIS_OK", 1: "PLIS_ERR_INVALID", 2: "PLIS_ERR_PARSE", 3: "PLIS_ERR_IO", 4: "PLIS_ERR_OOM",
    5: "PLIS_ERR_CUDA", 6: "PLIS_ERR_TIMEOUT", 7: "PLIS_ERR_STUCK", 8: "PLIS_ERR_OVERFLOW",
    9: "PLIS_ERR_LIMIT", 10: "PLIS_ERR_NO_DEVICE", 11: "PLIS_ERR_UNSUPPORTED",
}
MODE_REFERENCE, MODE_CORRECTED = 0, 1
PREC_FP64, PREC_FP32 = 0, 1
LEAP_CR, LEAP_NOCR, SSA, SSA_FF = 0, 1, 2, 3
STOP_NONE, STOP_TIME, STOP_STEPS, STOP_NO_EVENT, STOP_ERROR = 0, 1, 2, 3, 4


class ModelDesc(ctypes.Structure):
    _fields_ = [("n_subvolumes", u32), ("n_species", u32), ("n_reactions", u32), ("n_compartments", u32),
                ("neighbours", vp), ("lattice_x", u32), ("lattice_y", u32), ("lattice_z", u32),
                ("reactants", vp), ("products", vp), ("reaction_rates", vp), ("diffusion_rates", vp),
                ("compartment", vp)]


class Options(ctypes.Structure):
    _fields_ = [("size", u32), ("mode", i32), ("precision", i32), ("critical_threshold", i32),
                ("epsilon", f64), ("seed", u64), ("replica", u32), ("device", i32), ("max_rollbacks", i32),
                ("steps_per_launch", i32), ("tile", i32 * 3), ("persistent", i32), ("profile", i32),
                ("stage_halo", i32), ("learned_mlp", i32), ("wait_polls", u64), ("pooled_draws", i32)]


class Profile(ctypes.Structure):
    _fields_ = [("ms", f64 * 4), ("launches", u64 * 4)]


KERNEL_NAMES = ("leap", "exact", "apply", "classify")


class Stats(ctypes.Structure):
    _fields_ = [("time", f64), ("steps", u64), ("rollbacks", u64), ("events", u64), ("exact_events", u64),
                ("stop_reason", i32), ("status", i32), ("last_tau", f64), ("last_argmin", i64),
                ("device_ms", f64), ("kernel_launches", u64)]


class SlabBuffers(ctypes.Structure):
    _fields_ = [("send", vp * 2), ("recv", vp * 2), ("stage_words", u64), ("summary", vp), ("summary_all", vp),
                ("summary_bytes", u64), ("remote", vp), ("remote_all", vp), ("remote_bytes", u64)]


class BatchDesc(ctypes.Structure):
    _fields_ = [("n_replicas", u32), ("n_species", u32), ("n_reactions", u32), ("reactants", vp), ("products", vp),
                ("lattice", vp), ("reaction_rates", vp), ("diffusion_rates", vp), ("replica_ids", vp)]


class BatchTuning(ctypes.Structure):
    _fields_ = [("tile", i32 * 3), ("blocks_per_sm", i32), ("grid", i32), ("events_per_s", f64)]


class TrainParams(ctypes.Structure):
    _fields_ = [("iterations", u64), ("batch", u32), ("learning_rate", ctypes.c_float), ("quantile", ctypes.c_float),
                ("seed", u64)]


class TrainReport(ctypes.Structure):
    _fields_ = [("loss_first", f64), ("loss_last", f64), ("records", u64), ("iterations", u64), ("device_ms", f64)]


PROPOSER_WEIGHTS = 8977
# plis_trace_record (64 bytes)
import numpy as _np  # noqa: E402

TRACE_DTYPE = _np.dtype([("features", "<f4", (8,)), ("tau_cao", "<f4"), ("tau_step", "<f4"), ("label", "<f4"),
                         ("subvolume", "<u4"), ("counts", "<i4", (4,))])
assert TRACE_DTYPE.itemsize == 64
# plis_event_record (32 bytes) and its kinds
EVENT_DTYPE = _np.dtype([("time", "<f8"), ("step", "<u8"), ("subvolume", "<u4"), ("target", "<u4"),
                         ("count", "<u4"), ("channel", "<u2"), ("kind", "u1"), ("attempt", "u1")])
assert EVENT_DTYPE.itemsize == 32
EVENT_KINDS = {1: "leap_reaction", 2: "leap_diffusion", 3: "critical_reaction", 4: "critical_diffusion",
               5: "ssa_reaction", 6: "ssa_diffusion"}


class ConfigView(ctypes.Structure):
    _fields_ = [("model", ModelDesc), ("initial_state", vp), ("end_time", f64), ("log_freq", f64)]


class PlisError(RuntimeError):
    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")


def _load() -> ctypes.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python pliscuda_b200/build.py`")
    lib = ctypes.CDLL(LIB_PATH)
    P = ctypes.POINTER
    sig = {
        "plis_abi_version": (i32, []),
        "plis_last_error": (ctypes.c_char_p, []),
        "plis_status_string": (ctypes.c_char_p, [i32]),
        "plis_options_init": (None, [P(Options)]),
        "plis_create": (i32, [P(ModelDesc), P(Options), P(vp)]),
        "plis_destroy": (i32, [vp]),
        "plis_set_state": (i32, [vp, vp]),
        "plis_get_state": (i32, [vp, vp]),
        "plis_set_time": (i32, [vp, f64]),
        "plis_set_state_at": (i32, [vp, vp, f64, u64]),
        "plis_slab_setup": (i32, [vp, u32, u32, u32, u32]),
        "plis_slab_buffers_get": (i32, [vp, vp]),
        "plis_slab_phase": (i32, [vp, i32, f64, u64]),
        "plis_run": (i32, [vp, f64]),
        "plis_step": (i32, [vp, u64]),
        "plis_get_stats": (i32, [vp, P(Stats)]),
        "plis_get_taus": (i32, [vp, vp, vp]),
        "plis_set_event_log": (i32, [vp, u64]),
        "plis_read_event_log": (i32, [vp, vp, u64, P(u64), P(u64), i32]),
        "plis_get_profile": (i32, [vp, P(Profile)]),
        "plis_tau_argmin_noalloc": (i32, [vp, u64, vp, vp, vp]),
        "plis_batch_create": (i32, [P(BatchDesc), P(Options), P(vp)]),
        "plis_batch_destroy": (i32, [vp]),
        "plis_batch_set_state": (i32, [vp, u32, vp]),
        "plis_batch_get_state": (i32, [vp, u32, vp]),
        "plis_batch_get_taus": (i32, [vp, u32, vp, vp]),
        "plis_batch_run": (i32, [vp, f64]),
        "plis_batch_step": (i32, [vp, u64]),
        "plis_batch_get_stats": (i32, [vp, u32, P(Stats)]),
        "plis_batch_autotune": (i32, [vp, u64, P(BatchTuning)]),
        "plis_batch_get_tuning": (i32, [vp, P(BatchTuning)]),
        "plis_batch_set_proposer": (i32, [vp, vp, f64]),
        "plis_canonical_neighbours": (i32, [u32, vp, vp, vp, vp]),
        "plis_config_load": (i32, [ctypes.c_char_p, P(vp)]),
        "plis_config_view_get": (i32, [vp, P(ConfigView)]),
        "plis_config_free": (None, [vp]),
        "plis_parse_topology": (i32, [ctypes.c_char_p, P(u32), P(vp)]),
        "plis_parse_state": (i32, [ctypes.c_char_p, P(u32), P(u32), P(vp)]),
        "plis_parse_reactions": (i32, [ctypes.c_char_p, P(u32), P(u32), P(vp), P(vp)]),
        "plis_free": (None, [vp]),
        "plis_write_snapshot": (i32, [ctypes.c_char_p, vp, u32, u32, f64]),
        "plis_run_simulation": (i32, [P(ModelDesc), vp, f64, f64, f64, P(Options), ctypes.c_char_p, i32, P(Stats)]),
        "plis_read_snapshot": (i32, [ctypes.c_char_p, P(u32), P(u32), P(f64), P(vp)]),
        "plis_train_params_init": (None, [P(TrainParams)]),
        "plis_learner_create": (i32, [u64, i32, P(vp)]),
        "plis_learner_destroy": (i32, [vp]),
        "plis_learner_record": (i32, [vp, vp, u64, u32, f64]),
        "plis_learner_count": (i32, [vp, P(u64)]),
        "plis_learner_get_records": (i32, [vp, u64, u64, vp]),
        "plis_learner_set_records": (i32, [vp, vp, u64]),
        "plis_learner_train": (i32, [vp, P(TrainParams), P(TrainReport)]),
        "plis_learner_gradient": (i32, [vp, ctypes.c_float, vp, P(f64)]),
        "plis_learner_predict": (i32, [vp, vp, u64, vp, i32]),
        "plis_learner_get_weights": (i32, [vp, vp]),
        "plis_learner_set_weights": (i32, [vp, vp]),
        "plis_set_proposer": (i32, [vp, vp, f64]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.plis_abi_version() != 1:
        raise ImportError("libplis.so ABI version mismatch")
    return lib


lib = _load()


def check(status: int) -> None:
    if status != PLIS_OK:
        raise PlisError(status, (lib.plis_last_error() or b"").decode(errors="replace"))


def default_options(**kw) -> Options:
    o = Options()
    lib.plis_options_init(ctypes.byref(o))
    for k, v in kw.items():
        if k == "tile":
            for i in range(3):
                o.tile[i] = int(v[i])
        else:
            setattr(o, k, v)
    return o
