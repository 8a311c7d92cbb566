"""ctypes access to the CPU oracle (oracle/_build/liboracle.so) for the tests.

The oracle is the checker: tests compare the engine's results with it. Nothing in the
product imports this module.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
ORACLE_DIR = ROOT / "oracle"
LIB = ORACLE_DIR / "_build" / "liboracle.so"
CLI = ORACLE_DIR / "_build" / "axon_oracle"
U32P = C.POINTER(C.c_uint32)

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


class OracleCfg(C.Structure):
    """The network configuration struct of include/axon_capi.h, declared here so that the
    oracle can be driven without loading the engine library."""
    _fields_ = [(f, C.c_uint32) for f in CFG_FIELDS] + [("reserved", C.c_uint32 * 9)]


_lib = None


def default_threads() -> int:
    """Host threads for an oracle run: AXON_ORACLE_THREADS, else every core."""
    import os

    return int(os.environ.get("AXON_ORACLE_THREADS", "0")) or (os.cpu_count() or 1)


def build() -> None:
    subprocess.run(["make", "-s", "-C", str(ORACLE_DIR)], check=True)


def load():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(str(LIB))
        L.oracle_create.restype = C.c_void_p
        L.oracle_create.argtypes = [C.c_void_p, C.c_uint]
        L.oracle_destroy.argtypes = [C.c_void_p]
        L.oracle_init.argtypes = [C.c_void_p, C.c_uint32]
        L.oracle_present.argtypes = [C.c_void_p, U32P, C.c_uint32, C.c_uint32, C.c_int, C.c_int, C.c_uint32]
        L.oracle_buf_words.restype = C.c_uint64
        L.oracle_buf_words.argtypes = [C.c_void_p, C.c_int]
        L.oracle_read.argtypes = [C.c_void_p, C.c_int, U32P, C.c_uint64]
        L.oracle_write.argtypes = [C.c_void_p, C.c_int, U32P, C.c_uint64]
        L.oracle_wstat.restype = C.c_uint32
        L.oracle_wstat.argtypes = [C.c_void_p]
        L.oracle_within.argtypes = [C.c_void_p, U32P, C.c_uint32, U32P, U32P, U32P]
        L.oracle_indeg.argtypes = [C.c_void_p, U32P]
        L.oracle_untouched.argtypes = [C.c_void_p, U32P]
        L.oracle_wdiag.argtypes = [C.c_void_p, U32P, U32P, C.c_uint32, C.c_uint32, U32P]
        L.oracle_bstest.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, U32P, U32P, U32P, U32P, U32P, C.c_uint64]
        L.oracle_kwtatest.argtypes = [U32P, U32P, U32P, C.c_uint32]
        L.oracle_stimuli.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, U32P]
        L.oracle_load_stim.argtypes = [U32P, C.c_uint32, C.c_double, C.c_uint32, C.c_uint32, U32P]
        L.oracle_uniform_int.argtypes = [C.c_uint32, C.c_uint64, C.c_uint64, C.c_uint32, C.POINTER(C.c_uint64)]
        L.oracle_canonical.argtypes = [C.c_uint32, C.c_uint32, C.POINTER(C.c_double)]
        L.oracle_noisy_cue.argtypes = [U32P, C.c_uint32, C.c_double, C.c_uint32, C.c_uint32, U32P]
        L.oracle_noisy_seed.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32]
        L.oracle_noisy_seed.restype = C.c_uint32
        L.oracle_cfg.argtypes = [C.c_int, C.POINTER(C.c_char_p), C.c_void_p]
        _lib = L
    return _lib


def u32(a: np.ndarray):
    assert a.dtype == np.uint32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(U32P)


class OracleNet:
    """CPU restatement with the same calls as axon_b200.Network."""

    def __init__(self, cfg, threads: int = 8):
        self.L = load()
        self.cfg = cfg
        self.ncol = cfg.ncol
        self.n = cfg.ncol * 32
        self._h = self.L.oracle_create(C.byref(cfg), threads)

    def close(self):
        if self._h:
            self.L.oracle_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def init(self, seed: int):
        self.L.oracle_init(self._h, seed)

    def present(self, stim, T, clamp_steps, learn, freeze=False, use_bias=2):
        stim = np.ascontiguousarray(stim, dtype=np.uint32)
        self.L.oracle_present(self._h, u32(stim), T, clamp_steps, int(learn), int(freeze), use_bias)

    def read(self, name: str) -> np.ndarray:
        n = self.L.oracle_buf_words(self._h, BUF[name])
        out = np.empty(n, dtype=np.uint32)
        assert self.L.oracle_read(self._h, BUF[name], u32(out), n) == 0
        return out

    def write(self, name: str, arr: np.ndarray):
        arr = np.ascontiguousarray(arr, dtype=np.uint32)
        assert self.L.oracle_write(self._h, BUF[name], u32(arr), arr.size) == 0

    def wstat(self) -> int:
        return int(self.L.oracle_wstat(self._h))

    def within(self, ball, use_mask=0, post_mask=None, mult=None):
        out = np.zeros(10, dtype=np.uint32)
        ball = np.ascontiguousarray(ball, dtype=np.uint32)
        pm = u32(np.ascontiguousarray(post_mask, dtype=np.uint32)) if post_mask is not None else None
        mu = u32(np.ascontiguousarray(mult, dtype=np.uint32)) if mult is not None else None
        self.L.oracle_within(self._h, u32(ball), use_mask, pm, mu, u32(out))
        return out

    def indeg(self):
        out = np.empty(self.n, dtype=np.uint32)
        self.L.oracle_indeg(self._h, u32(out))
        return out

    def untouched(self):
        out = np.empty(self.n, dtype=np.uint32)
        self.L.oracle_untouched(self._h, u32(out))
        return out

    def wdiag(self, memb, asm_spk, nstim, sel):
        out = np.zeros(48, dtype=np.uint32)
        self.L.oracle_wdiag(self._h, u32(np.ascontiguousarray(memb, dtype=np.uint32)),
                            u32(np.ascontiguousarray(asm_spk, dtype=np.uint32)), nstim, sel, u32(out))
        return out


def config(**kw) -> OracleCfg:
    """The reference's built-in defaults as the oracle's own key parser restates them
    (src/axon.mm:688-735), with CLI keys overridden by ``kw`` (key=value, as on the command
    line; e.g. config(ncol=4096, target=64))."""
    args = [f"{k}={int(v)}".encode() for k, v in kw.items()]
    argv = (C.c_char_p * max(1, len(args)))(*args)
    c = OracleCfg()
    load().oracle_cfg(len(args), argv, C.byref(c))
    return c


def noisy_cue(cols, frac, seed, ncol) -> np.ndarray:
    cols = np.ascontiguousarray(cols, dtype=np.uint32)
    out = np.empty(ncol, dtype=np.uint32)
    load().oracle_noisy_cue(u32(cols), cols.size, frac, seed, ncol, u32(out))
    return out


def noisy_seed(q, pct, draw) -> int:
    return int(load().oracle_noisy_seed(q, pct, draw))


def stimuli(seed, nstim, incols, stimcols) -> np.ndarray:
    out = np.empty(nstim * stimcols, dtype=np.uint32)
    load().oracle_stimuli(seed, nstim, incols, stimcols, u32(out))
    return out.reshape(nstim, stimcols)


def load_stim(cols, keep, seed, ncol) -> np.ndarray:
    cols = np.ascontiguousarray(cols, dtype=np.uint32)
    out = np.empty(ncol, dtype=np.uint32)
    load().oracle_load_stim(u32(cols), cols.size, keep, seed, ncol, u32(out))
    return out


def bstest(op, lo, hi, planes, mask):
    ps = [np.ascontiguousarray(p, dtype=np.uint32) for p in planes]
    m = np.ascontiguousarray(mask, dtype=np.uint32)
    load().oracle_bstest(op, lo, hi, *(u32(p) for p in ps), u32(m), m.size)
    return ps


def kwtatest(values, ks):
    """The oracle's k-of-32 ranking on (n, 32) values: (n, 3) = ballot, vk, vk1."""
    v = np.ascontiguousarray(values, dtype=np.uint32)
    k = np.ascontiguousarray(ks, dtype=np.uint32)
    out = np.zeros((k.size, 3), dtype=np.uint32)
    load().oracle_kwtatest(u32(v), u32(k), u32(out), k.size)
    return out


def run_cli(args: list[str], threads: int | None = None, timeout: float = 3600) -> str:
    import os

    load()
    env = dict(os.environ)
    if threads:
        env["AXON_ORACLE_THREADS"] = str(threads)
    p = subprocess.run([str(CLI), *args], capture_output=True, text=True, env=env, timeout=timeout)
    if p.returncode != 0:
        raise RuntimeError(p.stderr)
    return p.stdout
