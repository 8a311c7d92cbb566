"""Python mirror of the reference's engine state machine over the C ABI.

``Network`` holds one AXON network on a GPU. Its methods are the reference's device
operations (src/axon.mm): ``init`` = k_init_w + k_init_conn, ``present`` = present(),
``wstat`` = k_wstat, ``within`` = k_within, ``indeg`` = k_indeg, ``untouched`` =
k_untouched, ``wdiag`` = k_wdiag. Buffers are read and written by the reference's
MTLBuffer names (``read("W3")``, ``write("REFBALL", ...)``).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi as A


def config(**kw) -> A.AxonCfg:
    """Reference CLI defaults (src/axon.mm:688-731) overridden by ``kw`` (CLI key names)."""
    return A.default_cfg(**kw)


CONFIG_C = dict(nand=4, target=64, k=24, dthr=1, mode=1, inbr=4, contrast=1, margingate=0, ltdrep=1,
                ltdevery=2, biasup=73, biasdown=1)


class Network:
    def __init__(self, cfg: A.AxonCfg | dict | None = None, device: int = 0):
        if cfg is None or isinstance(cfg, dict):
            cfg = config(**(cfg or {}))
        self.cfg = cfg
        self.ncol = cfg.ncol
        self.n = cfg.ncol * 32
        h = C.c_void_p()
        A.check(A.lib().axon_create(C.byref(cfg), device, C.byref(h)))
        self._h = h

    def close(self) -> None:
        if self._h:
            A.lib().axon_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- state machine
    def init(self, seed: int) -> None:
        A.check(A.lib().axon_init(self._h, seed))

    def present(self, stim: np.ndarray, T: int, clamp_steps: int, learn: bool, freeze: bool = False,
                use_bias: int = 2) -> float:
        stim = np.ascontiguousarray(stim, dtype=np.uint32)
        assert stim.shape == (self.ncol,)
        ms = C.c_double()
        A.check(A.lib().axon_present(self._h, A.u32(stim), T, clamp_steps, int(learn), int(freeze), use_bias,
                                     C.byref(ms)))
        return ms.value

    def clone(self) -> "Network":
        """A second network with a copy of every device buffer of this one."""
        other = Network.__new__(Network)
        other.cfg, other.ncol, other.n = self.cfg, self.ncol, self.n
        h = C.c_void_p()
        A.check(A.lib().axon_clone(self._h, C.byref(h)))
        other._h = h
        return other

    def profile_present(self, stim: np.ndarray, T: int, clamp_steps: int, learn: bool = True,
                        use_bias: int = 2) -> dict:
        """One presentation timed per phase with the device timer (us per step)."""
        stim = np.ascontiguousarray(stim, dtype=np.uint32)
        out = (C.c_double * 6)()
        A.check(A.lib().axon_profile_present(self._h, A.u32(stim), T, clamp_steps, int(learn), use_bias, out))
        return {"drive_us": out[0], "barrier_us": out[1], "emit_us": out[2], "learn_us": out[3], "step_us": out[4],
                "launch_ms": out[5]}

    def set_wait_limit(self, ns: int) -> None:
        A.check(A.lib().axon_set_wait_limit(self._h, ns))

    def inject_missing_arrival(self, missing: int = 1) -> None:
        """Failure-detection hook: the next persistent launch waits for absent CTAs."""
        A.check(A.lib().axon_inject_missing_arrival(self._h, missing))

    # -- checkpoints
    def save(self, path: str, seed: int, nstim: int, stimcols: int, epochs: int) -> None:
        """Writes the trained state (W0..W3, conn, bias, mult) and its metadata to `path`."""
        m = A.CkptMeta(seed=seed, nstim=nstim, stimcols=stimcols, epochs=epochs)
        A.check(A.lib().axon_save(self._h, str(path).encode(), C.byref(m)))

    def load(self, path: str) -> dict:
        """Replaces the state with a checkpoint's (same configuration required); returns its metadata."""
        m = A.CkptMeta()
        A.check(A.lib().axon_load(self._h, str(path).encode(), C.byref(m)))
        return {"seed": m.seed, "nstim": m.nstim, "stimcols": m.stimcols, "epochs": m.epochs}

    # -- buffers
    def words(self, name: str) -> int:
        return int(A.lib().axon_buf_words(self._h, A.BUF[name]))

    def read(self, name: str) -> np.ndarray:
        out = np.empty(self.words(name), dtype=np.uint32)
        A.check(A.lib().axon_read(self._h, A.BUF[name], A.u32(out), out.size))
        return out

    def write(self, name: str, arr: np.ndarray) -> None:
        arr = np.ascontiguousarray(arr, dtype=np.uint32)
        A.check(A.lib().axon_write(self._h, A.BUF[name], A.u32(arr), arr.size))

    def recall(self, cues: np.ndarray, T: int, clamp_steps: int, use_bias: int = 0, method: str = "batched",
               hist: bool = False, stats: bool = False, ref_ball: np.ndarray | None = None,
               drive_log: np.ndarray | None = None, graph: bool = False, final_out: np.ndarray | None = None,
               contraction: str = "popc", slab: str = "floor") -> dict:
        """B readout trajectories (present() with learn=0 for each cue row) in one call.

        contraction: "popc" (CUDA cores) or "tensor" (binary MMA) computes the batched
        method's AND-popcounts; the results are the same.
        slab: which per-neuron drives the batched method stores for the k-of-32 of gated
        columns: "floor" (columns at or above the trajectory's histogram floor, all of them
        at the step after the clamp), "floor_always" or "full"; gated columns without a
        stored drive are recomputed, and the results are the same.

        Returns {"final": (B, ncol), "hist": (B, T, ncol) | None, "stats": (B, 1024) | None,
        "drive_log": (B, 256) | None, "gpu_ms": float}. final_out, a C-contiguous uint32
        (B, ncol) array (page-locked memory copies fastest), receives the final spikes in
        place of a new array.
        """
        cues = np.ascontiguousarray(cues, dtype=np.uint32)
        B = cues.shape[0]
        assert cues.shape == (B, self.ncol)
        a = A.RecallArgs(T=T, clamp_steps=clamp_steps, use_bias=use_bias,
                         method=A.RECALL_BATCHED if method == "batched" else A.RECALL_PLAIN, graph=int(graph),
                         contraction=A.CONTRACT_TENSOR if contraction == "tensor" else A.CONTRACT_POPC,
                         slab=A.SLAB[slab])
        if final_out is not None:
            assert final_out.dtype == np.uint32 and final_out.shape == (B, self.ncol) and final_out.flags.c_contiguous
        out = {"final": final_out if final_out is not None else np.empty((B, self.ncol), dtype=np.uint32),
               "hist": np.empty((B, T, self.ncol), dtype=np.uint32) if hist else None,
               "stats": np.empty((B, 1024), dtype=np.uint32) if stats else None,
               "drive_log": None}
        rb = None
        if ref_ball is not None:
            rb = np.ascontiguousarray(ref_ball, dtype=np.uint32)
            assert rb.shape == (B, self.ncol)
        if drive_log is not None or rb is not None:
            out["drive_log"] = (np.zeros((B, 256), dtype=np.uint32) if drive_log is None
                                else np.ascontiguousarray(drive_log, dtype=np.uint32).copy())
        ptr = lambda x: None if x is None else x.ctypes.data_as(C.c_void_p)  # noqa: E731
        ms = C.c_double()
        A.check(A.lib().axon_recall(self._h, ptr(cues), B, C.byref(a), ptr(rb), ptr(out["final"]), ptr(out["hist"]),
                                    ptr(out["stats"]), ptr(out["drive_log"]), C.byref(ms)))
        out["gpu_ms"] = ms.value
        return out

    def recall_device(self, cues_ptr: int, B: int, T: int, clamp_steps: int, final_ptr: int | None = None,
                      use_bias: int = 0, method: str = "batched", graph: bool = False,
                      contraction: str = "popc", slab: str = "floor") -> float:
        """Device-resident variant: cues/final are device addresses on this network's GPU.
        graph=True replays a captured CUDA graph of the launch while the arguments repeat."""
        a = A.RecallArgs(T=T, clamp_steps=clamp_steps, use_bias=use_bias,
                         method=A.RECALL_BATCHED if method == "batched" else A.RECALL_PLAIN, graph=int(graph),
                         contraction=A.CONTRACT_TENSOR if contraction == "tensor" else A.CONTRACT_POPC,
                         slab=A.SLAB[slab])
        ms = C.c_double()
        A.check(A.lib().axon_recall_device(self._h, C.c_void_p(cues_ptr), B, C.byref(a), None,
                                           None if final_ptr is None else C.c_void_p(final_ptr), None, None, None,
                                           C.byref(ms)))
        return ms.value

    def final_spikes(self, T: int) -> np.ndarray:
        """The spike buffer present() wrote last (spkB after an odd T, spkA after an even T)."""
        return self.read("SPK_B" if (T & 1) else "SPK_A")

    # -- diagnostics
    def wstat(self) -> int:
        v = C.c_uint32()
        A.check(A.lib().axon_wstat(self._h, C.byref(v)))
        return v.value

    def within(self, ball: np.ndarray, use_mask: int = 0, post_mask: np.ndarray | None = None,
               mult: np.ndarray | None = None) -> np.ndarray:
        ball = np.ascontiguousarray(ball, dtype=np.uint32)
        out = np.zeros(10, dtype=np.uint32)
        pm = A.u32(np.ascontiguousarray(post_mask, dtype=np.uint32)) if post_mask is not None else None
        mu = A.u32(np.ascontiguousarray(mult, dtype=np.uint32)) if mult is not None else None
        A.check(A.lib().axon_within(self._h, A.u32(ball), use_mask, pm, mu, A.u32(out)))
        return out

    def indeg(self) -> np.ndarray:
        out = np.empty(self.n, dtype=np.uint32)
        A.check(A.lib().axon_indeg(self._h, A.u32(out)))
        return out

    def untouched(self) -> np.ndarray:
        out = np.empty(self.n, dtype=np.uint32)
        A.check(A.lib().axon_untouched(self._h, A.u32(out)))
        return out

    def wdiag(self, memb: np.ndarray, asm_spk: np.ndarray, nstim: int, sel: int) -> np.ndarray:
        out = np.zeros(48, dtype=np.uint32)
        A.check(A.lib().axon_wdiag(self._h, A.u32(np.ascontiguousarray(memb, dtype=np.uint32)),
                                   A.u32(np.ascontiguousarray(asm_spk, dtype=np.uint32)), nstim, sel, A.u32(out)))
        return out


def multi_train(nets: list[Network], seeds: list[int], nstim: list[int], *, epochs: int, T: int = 10,
                clamp_steps: int = 5, train_clamp: int | None = None, stimcols: int = 64, wave_t: int = 35,
                readout: bool = True, autotune: bool = True, slots: int = 0, threads: int = 1024,
                graph: bool = True, method: str = "launch") -> tuple[list[dict], dict]:
    """The reference experiment for many networks at once (axon_multi_train).

    Every network is initialised from its seed and trained on its own load; all
    presentations run in one persistent launch (``method="launch"``) or through the plain
    path, one launch per presentation (``method="plain"``). Returns the per-network
    measurements and the launch report."""
    n = len(nets)
    assert len(seeds) == n and len(nstim) == n
    a = A.MultiArgs(epochs=epochs, T=T, clamp_steps=clamp_steps,
                    train_clamp=clamp_steps if train_clamp is None else train_clamp, stimcols=stimcols,
                    wave_t=wave_t, readout=int(readout), autotune=int(autotune), slots=slots, threads=threads,
                    graph=int(graph), method=A.MULTI_PLAIN if method == "plain" else A.MULTI_ONE_LAUNCH)
    hs = (C.c_void_p * n)(*[x._h for x in nets])
    sd = np.ascontiguousarray(seeds, dtype=np.uint32)
    ns = np.ascontiguousarray(nstim, dtype=np.uint32)
    res = (A.MultiResult * n)()
    rep = A.MultiReport()
    A.check(A.lib().axon_multi_train(hs, n, A.u32(sd), A.u32(ns), C.byref(a), res, C.byref(rep)))
    out = [{f: getattr(r, f) for f, _ in A.MultiResult._fields_} for r in res]
    return out, {f: getattr(rep, f) for f, _ in A.MultiReport._fields_}


def clock_s() -> float:
    """The monotonic host clock the server stamps requests with (seconds)."""
    return float(A.lib().axon_clock_s())


class Server:
    """Recall server over device-resident networks (axon_serve_*): requests are readout
    trajectories (cue columns clamped for ``clamp_steps``, then ``free_steps`` free steps)
    run with continuous batching on an internal thread of the library."""

    def __init__(self, nets: list[Network], mem_bytes: int = 64 << 20):
        self.nets = list(nets)
        self.ncol = nets[0].ncol
        hs = (C.c_void_p * len(nets))(*[x._h for x in nets])
        h = C.c_void_p()
        A.check(A.lib().axon_serve_create(hs, len(nets), mem_bytes, C.byref(h)))
        self._h = h

    def submit(self, net: int, cue_cols, clamp_steps: int, free_steps: int, tag: int, arrive_s: float = 0.0) -> None:
        cols = np.ascontiguousarray(cue_cols, dtype=np.uint32)
        A.check(A.lib().axon_serve_submit(self._h, net, A.u32(cols) if cols.size else None, cols.size, clamp_steps,
                                          free_steps, tag, arrive_s))

    def poll(self, max_results: int = 4096, spikes: bool = True) -> list[tuple[dict, np.ndarray | None]]:
        res = (A.ServeResult * max_results)()
        spk = np.empty((max_results, self.ncol), dtype=np.uint32) if spikes else None
        n = C.c_uint32()
        A.check(A.lib().axon_serve_poll(self._h, res, A.u32(spk) if spikes else None, max_results, C.byref(n)))
        return [({f: getattr(res[i], f) for f, _ in A.ServeResult._fields_}, spk[i].copy() if spikes else None)
                for i in range(n.value)]

    def wait_idle(self, timeout_s: float = 120.0) -> None:
        A.check(A.lib().axon_serve_wait_idle(self._h, timeout_s))

    def stats(self) -> dict:
        c = A.ServeCounters()
        A.check(A.lib().axon_serve_stats(self._h, C.byref(c)))
        return {f: getattr(c, f) for f, _ in A.ServeCounters._fields_}

    def close(self) -> None:
        if self._h:
            A.lib().axon_serve_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def clamp_words(cols, ncol: int) -> np.ndarray:
    """Clamp words with 0xFFFFFFFF on the given input columns (the reference's clamp form)."""
    w = np.zeros(ncol, dtype=np.uint32)
    w[np.asarray(cols, dtype=np.int64)] = 0xFFFFFFFF
    return w


def stimuli(seed: int, nstim: int, incols: int, stimcols: int) -> np.ndarray:
    """Input patterns of the reference protocol (src/axon.mm:793-799), shape (nstim, stimcols)."""
    out = np.empty(nstim * stimcols, dtype=np.uint32)
    A.check(A.lib().axon_stimuli(seed, nstim, incols, stimcols, A.u32(out)))
    return out.reshape(nstim, stimcols)


def load_stim(cols: np.ndarray, keep: float, seed: int, ncol: int) -> np.ndarray:
    """Clamp words of one presentation (loadStim, src/axon.mm:800-804)."""
    cols = np.ascontiguousarray(cols, dtype=np.uint32)
    out = np.empty(ncol, dtype=np.uint32)
    A.check(A.lib().axon_load_stim(A.u32(cols), cols.size, C.c_double(keep), seed, ncol, A.u32(out)))
    return out


def noisy_cue(cols: np.ndarray, frac: float, seed: int, ncol: int) -> np.ndarray:
    """Clamp words of the whole pattern with round(frac * 32 * len(cols)) of its active bits
    flipped off, chosen from a seeded stream (axon_noisy_cue)."""
    cols = np.ascontiguousarray(cols, dtype=np.uint32)
    out = np.empty(ncol, dtype=np.uint32)
    A.check(A.lib().axon_noisy_cue(A.u32(cols), cols.size, C.c_double(frac), seed, ncol, A.u32(out)))
    return out


def noisy_cue_seed(q: int, pct: int, draw: int) -> int:
    """Seed of draw `draw` of pattern q's noisy cue at `pct` percent flipped (axon_noisy_cue_seed)."""
    return int(A.lib().axon_noisy_cue_seed(q, pct, draw))


def kwtatest(values: np.ndarray, ks: np.ndarray, device: int = 0) -> np.ndarray:
    """Runs the kernels' k-of-32 on (n, 32) values with one k per row: (n, 3) = winners
    ballot, vk, vk1."""
    v = np.ascontiguousarray(values, dtype=np.uint32)
    k = np.ascontiguousarray(ks, dtype=np.uint32)
    assert v.shape == (k.size, 32)
    out = np.zeros((k.size, 3), dtype=np.uint32)
    A.check(A.lib().axon_kwtatest(device, A.u32(v), A.u32(k), A.u32(out), k.size))
    return out


def bstest(op: int, lo: int, hi: int, planes: list[np.ndarray], mask: np.ndarray, device: int = 0) -> None:
    """Runs the bit-serial inc/dec/clip kernel in place on four planes (k_bstest)."""
    ps = [np.ascontiguousarray(p, dtype=np.uint32) for p in planes]
    m = np.ascontiguousarray(mask, dtype=np.uint32)
    A.check(A.lib().axon_bstest(device, op, lo, hi, *(A.u32(p) for p in ps), A.u32(m), m.size))
    for dst, src in zip(planes, ps):
        dst[...] = src
