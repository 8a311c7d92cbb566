"""ctypes binding of libaxon_b200.so (declarations in include/axon_capi.h).

The library is built in-tree by ``axon_b200.build``; if it is missing this module raises
instead of falling back to anything else: there is no CPU path in the product.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "_build" / "libaxon_b200.so"

AXON_OK, AXON_EINVAL, AXON_ENOMEM, AXON_ECUDA, AXON_ETIMEOUT, AXON_ESTATE = range(6)

BUF = {
    "W0": 0, "W1": 1, "W2": 2, "W3": 3, "CONN": 4, "SPK_A": 5, "SPK_B": 6, "DRIVE": 7, "BBITS": 8,
    "ACC": 9, "BIAS": 10, "MARG": 11, "REFBALL": 12, "DRIVELOG": 13, "MULT": 14, "STIM": 15,
    "STATS": 16, "HIST": 17, "THETA": 18,
}

CFG_FIELDS = [
    "ncol", "incols", "inbr", "nand", "target", "k", "ktest", "dthr", "boost", "mode", "biasup",
    "biasdown", "biasshift", "biasdownevery", "bandlo", "bandhi", "contrast", "margingate", "hetero",
    "ltdrep", "ltdevery", "facil", "topkpar",
]


class AxonCfg(C.Structure):
    _fields_ = [(f, C.c_uint32) for f in CFG_FIELDS] + [("reserved", C.c_uint32 * 9)]


class RecallArgs(C.Structure):
    _fields_ = [("T", C.c_uint32), ("clamp_steps", C.c_uint32), ("use_bias", C.c_uint32), ("method", C.c_uint32),
                ("graph", C.c_uint32), ("contraction", C.c_uint32), ("slab", C.c_uint32), ("reserved", C.c_uint32 * 1)]


RECALL_BATCHED, RECALL_PLAIN = 0, 1
CONTRACT_POPC, CONTRACT_TENSOR = 0, 1
SLAB = {"floor": 0, "floor_always": 1, "full": 2}

STATE_DEV_FIELDS = ["w0", "w1", "w2", "w3", "conn", "bias", "mult", "refball", "stim", "spk_a", "spk_b", "drive",
                    "bbits", "acc", "marg", "drive_log", "stats", "hist", "theta"]


class StateDev(C.Structure):
    """Device pointers for axon_present_static (caller-owned buffers)."""
    _fields_ = [(f, C.c_void_p) for f in STATE_DEV_FIELDS]


MULTI_ARG_FIELDS = ["epochs", "T", "clamp_steps", "train_clamp", "stimcols", "wave_t", "readout", "autotune",
                    "slots", "threads", "graph", "method"]


class MultiArgs(C.Structure):
    _fields_ = [(f, C.c_uint32) for f in MULTI_ARG_FIELDS] + [("reserved", C.c_uint32 * 4)]


class MultiResult(C.Structure):
    _fields_ = [("within_pct", C.c_double), ("recall", C.c_double), ("best_other", C.c_double),
                ("drive_t6", C.c_double), ("wave_first", C.c_double), ("wave_last", C.c_double),
                ("wdens_pct", C.c_double), ("steps", C.c_uint64)]


class MultiReport(C.Structure):
    _fields_ = [("gpu_ms", C.c_double), ("tune_ms", C.c_double), ("steps", C.c_uint64), ("train_steps", C.c_uint64),
                ("slots", C.c_uint32), ("threads", C.c_uint32), ("tiles", C.c_uint32), ("grid", C.c_uint32),
                ("graph", C.c_uint32), ("tried", C.c_uint32), ("w3_tiles", C.c_uint64), ("learn_tasks", C.c_uint64)]


MULTI_ONE_LAUNCH, MULTI_PLAIN = 0, 1


class CkptMeta(C.Structure):
    _fields_ = [("seed", C.c_uint32), ("nstim", C.c_uint32), ("stimcols", C.c_uint32), ("epochs", C.c_uint32),
                ("reserved", C.c_uint32 * 4)]


class ServeResult(C.Structure):
    _fields_ = [("tag", C.c_uint64), ("net", C.c_uint32), ("steps", C.c_uint32), ("arrive_s", C.c_double),
                ("admit_s", C.c_double), ("done_s", C.c_double)]


class ServeCounters(C.Structure):
    _fields_ = [("slots", C.c_uint32), ("in_flight", C.c_uint32), ("queued", C.c_uint64), ("ticks", C.c_uint64),
                ("completed", C.c_uint64), ("max_batch", C.c_uint64), ("mean_batch", C.c_double),
                ("busy_s", C.c_double), ("drive_s", C.c_double), ("emit_s", C.c_double), ("slot_bytes", C.c_uint64),
                ("fixed_bytes", C.c_uint64)]


class AxonError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"axon status {status}: {msg}")
        self.status = status


_lib = None
U32P = C.POINTER(C.c_uint32)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is not built; run `python -m axon_b200.build`")
        L = C.CDLL(str(LIB_PATH))
        L.axon_cfg_defaults.argtypes = [C.POINTER(AxonCfg)]
        L.axon_last_error.restype = C.c_char_p
        L.axon_create.argtypes = [C.POINTER(AxonCfg), C.c_int, C.POINTER(C.c_void_p)]
        L.axon_destroy.argtypes = [C.c_void_p]
        L.axon_init.argtypes = [C.c_void_p, C.c_uint32]
        L.axon_present.argtypes = [C.c_void_p, U32P, C.c_uint32, C.c_uint32, C.c_int, C.c_int, C.c_uint32,
                                   C.POINTER(C.c_double)]
        L.axon_read.argtypes = [C.c_void_p, C.c_int, U32P, C.c_uint64]
        L.axon_write.argtypes = [C.c_void_p, C.c_int, U32P, C.c_uint64]
        L.axon_buf_words.argtypes = [C.c_void_p, C.c_int]
        L.axon_buf_words.restype = C.c_uint64
        L.axon_wstat.argtypes = [C.c_void_p, U32P]
        L.axon_within.argtypes = [C.c_void_p, U32P, C.c_uint32, U32P, U32P, U32P]
        L.axon_indeg.argtypes = [C.c_void_p, U32P]
        L.axon_untouched.argtypes = [C.c_void_p, U32P]
        L.axon_wdiag.argtypes = [C.c_void_p, U32P, U32P, C.c_uint32, C.c_uint32, U32P]
        L.axon_bstest.argtypes = [C.c_int, C.c_uint32, C.c_uint32, C.c_uint32, U32P, U32P, U32P, U32P, U32P,
                                  C.c_uint64]
        L.axon_kwtatest.argtypes = [C.c_int, U32P, U32P, U32P, C.c_uint32]
        L.axon_set_wait_limit.argtypes = [C.c_void_p, C.c_uint64]
        L.axon_clone.argtypes = [C.c_void_p, C.POINTER(C.c_void_p)]
        L.axon_profile_present.argtypes = [C.c_void_p, U32P, C.c_uint32, C.c_uint32, C.c_int, C.c_uint32,
                                           C.POINTER(C.c_double)]
        L.axon_inject_missing_arrival.argtypes = [C.c_void_p, C.c_uint32]
        L.axon_stimuli.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, U32P]
        L.axon_load_stim.argtypes = [U32P, C.c_uint32, C.c_double, C.c_uint32, C.c_uint32, U32P]
        L.axon_noisy_cue.argtypes = [U32P, C.c_uint32, C.c_double, C.c_uint32, C.c_uint32, U32P]
        L.axon_noisy_cue_seed.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32]
        L.axon_noisy_cue_seed.restype = C.c_uint32
        L.axon_present_static.argtypes = [C.POINTER(AxonCfg), C.POINTER(StateDev), C.c_uint32, C.c_uint32, C.c_int,
                                          C.c_uint32]
        L.axon_multi_train.argtypes = [C.POINTER(C.c_void_p), C.c_uint32, U32P, U32P, C.POINTER(MultiArgs),
                                       C.POINTER(MultiResult), C.POINTER(MultiReport)]
        L.axon_save.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(CkptMeta)]
        L.axon_load.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(CkptMeta)]
        L.axon_clock_s.restype = C.c_double
        L.axon_serve_create.argtypes = [C.POINTER(C.c_void_p), C.c_uint32, C.c_uint64, C.POINTER(C.c_void_p)]
        L.axon_serve_submit.argtypes = [C.c_void_p, C.c_uint32, U32P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64,
                                        C.c_double]
        L.axon_serve_poll.argtypes = [C.c_void_p, C.POINTER(ServeResult), U32P, C.c_uint32, C.POINTER(C.c_uint32)]
        L.axon_serve_wait_idle.argtypes = [C.c_void_p, C.c_double]
        L.axon_serve_stats.argtypes = [C.c_void_p, C.POINTER(ServeCounters)]
        L.axon_serve_destroy.argtypes = [C.c_void_p]
        for fn in (L.axon_recall, L.axon_recall_device):
            fn.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.POINTER(RecallArgs), C.c_void_p, C.c_void_p,
                           C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_double)]
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != AXON_OK:
        raise AxonError(status, lib().axon_last_error().decode(errors="replace"))


def u32(a: np.ndarray):
    assert a.dtype == np.uint32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(U32P)


def default_cfg(**kw) -> AxonCfg:
    c = AxonCfg()
    lib().axon_cfg_defaults(C.byref(c))
    for k, v in kw.items():
        setattr(c, k, int(v))
    return c
