"""Benchmark: batched recall on one trained AXON network, synaptic events/s on B200.

Workload (the batched-recall configuration): config C network (131,072 neurons, 512 MiB of
4-bit counters), 60 patterns, seed 0, trained for 40 epochs by the plain GPU path (setup,
untimed). 300 cues = the 60 whole stored patterns plus, for each fraction 10 % and 25 % and
two seeded draws each, the patterns with that fraction of their active cue bits flipped off
(axon_noisy_cue). Every trajectory is 10 clamped + 35 free steps with the intrinsic bias off
(the reference's readout setting). One bench step = one batched recall of all 300
trajectories. The trained planes and all 300 trajectories are checked against the CPU
oracle's answer for this workload (tests/golden/recall_load60.json).

Synaptic event: one presynaptic spike delivered to one postsynaptic neuron through conn,
i.e. per step sum over (column, branch) of 32 * popcount(spikes of the branch's group at
t-1). The count is fixed by the workload (identical for every method and for the oracle).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl axon|reference]
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

NCOL, INCOLS, STIMCOLS, LOAD, EPOCHS, SEED = 4096, 512, 64, 60, 40, 0
T_RECALL, CLAMP_RECALL = 45, 10
T_WAVE, CLAMP_WAVE = 35, 5  # the reference's wave readout: 5 clamped + 30 free steps
FLIP_PCTS, DRAWS = (10, 25), 2
L2_BYTES = 126 * 2 ** 20
GOLDEN = ROOT / "tests" / "golden" / "recall_load60.json"
PUBLISHED = ROOT / "tests" / "golden" / "published.json"
# config C as CLI keys (bench/cap10.sh:7)
CONFIG_C_KEYS = dict(nand=4, target=64, k=24, dthr=1, mode=1, inbr=4, contrast=1, margingate=0, ltdrep=1, ltdevery=2,
                     biasup=73, biasdown=1)


def make_cues(pats: np.ndarray, noisy_cue, noisy_seed) -> np.ndarray:
    """The 300 cues in batch order: the 60 whole patterns, then per fraction and draw the 60
    noisy ones (noisy_cue / noisy_seed from the engine's C ABI, or the oracle's)."""
    cues = [noisy_cue(pats[q], 0.0, 0, NCOL) for q in range(LOAD)]
    for pct in FLIP_PCTS:
        for d in range(DRAWS):
            cues += [noisy_cue(pats[q], pct / 100.0, noisy_seed(q, pct, d), NCOL) for q in range(LOAD)]
    return np.stack(cues)


def digest(*arrays: np.ndarray, n: int | None = None) -> str:
    """SHA-256 of the arrays' words (little-endian), as the fixture records them."""
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a, dtype="<u4").tobytes())
    return h.hexdigest()[:n] if n else h.hexdigest()


def fixture() -> dict | None:
    return json.loads(GOLDEN.read_text()) if GOLDEN.exists() else None


def check_against_fixture(fx: dict | None, idx, hists) -> dict:
    """Trajectories idx (their (T, ncol) spike histories) against the oracle's fixture."""
    if fx is None:
        return {"checked": 0, "mismatches": None, "source": "fixture missing"}
    rows = fx["trajectories"]
    idx = [int(b) for b in idx]
    bad = [b for b, h in zip(idx, hists) if digest(h, n=16) != rows[b]["hist"] or digest(h[-1], n=16) != rows[b]["final"]]
    return {"checked": len(idx), "mismatches": len(bad), "first_mismatch": bad[0] if bad else None,
            "source": "tests/golden/recall_load60.json (CPU oracle)"}


def events_per_step(hist: np.ndarray, conn: np.ndarray) -> np.ndarray:
    """Synaptic events of every (trajectory, step) from the spike history (B, T, ncol)."""
    ngrp = NCOL // 8
    fan = np.bincount(conn.astype(np.int64), minlength=ngrp).astype(np.float64)  # (col, branch) per group
    pc = np.bitwise_count(hist).reshape(hist.shape[0], hist.shape[1], ngrp, 8).sum(-1, dtype=np.int64)
    ev = np.zeros(hist.shape[:2], dtype=np.float64)
    ev[:, 1:] = 32.0 * (pc[:, :-1] * fan).sum(-1)
    return ev


def train(net, pats, load_stim) -> float:
    """The reference's training schedule (src/axon.mm:1009-1033) on `net` (engine or oracle)."""
    t0 = time.time()
    for _ in range(EPOCHS):
        for p in range(LOAD):
            net.present(load_stim(pats[p], 1.0, 1000 + p, NCOL), 10, 5, True)
    net.present(load_stim(pats[0], 1.0, 31337, NCOL), 10, 5, True)  # the reference's extra presentation
    return time.time() - t0


def trained_digest(net) -> str:
    return digest(*(net.read(n) for n in ("W0", "W1", "W2", "W3", "BIAS")))


MULTI_SEEDS, MULTI_LOADS = (0, 1, 2, 3, 4), (12, 24, 36, 48, 60)


def config_c():
    import axon_b200 as ax

    return ax.config(ncol=NCOL, incols=INCOLS, **ax.CONFIG_C)


def printed(r: dict) -> dict:
    """One network's measurements as the command line prints them."""
    first, last = float(f"{r['wave_first']:.3f}"), float(f"{r['wave_last']:.3f}")
    return {"within": f"{r['within_pct']:.2f}", "within_pct": f"{r['within_pct']:.4f}", "recall": f"{r['recall']:.3f}",
            "best_other": f"{r['best_other']:.3f}", "margin": f"{r['recall'] - r['best_other']:+.3f}",
            "sustained": f"{last / first:.3f}", "drive": f"{r['drive_t6']:.0f}"}


def published() -> dict:
    return json.loads(PUBLISHED.read_text())


def table1_equal(rows: dict) -> dict:
    """Per load: do the printed measurements equal the published Table 1 row?"""
    gold = {r["stim"]: r for r in published()["table1"]}
    keys = ("within", "recall", "best_other", "margin", "sustained", "drive")
    return {str(L): all(m[k] == gold[L][k] for k in keys) for L, m in rows.items() if L in gold}


def bench_multi(dev: int, nnets: int = 25, epochs: int = EPOCHS, pins: bool = True) -> dict:
    """25 networks of uneven load (seeds 0-4 x loads 12..60, config C, 40 epochs plus the
    readouts of the five measurements): one persistent launch with an autotuned shape,
    against the plain path running the same presentations one launch each. The seed-0
    rows are compared with the published Table 1 and the five-seed summaries with Table 2
    (its load 42 from five more networks, outside the timed workload), and seed-0 networks
    at Table 1's higher loads are trained and compared too (140 and 200, the loads of the
    serving networks, in one launch; 74, 90 and 300 through the plain path)."""
    import axon_b200 as ax
    from tests.metrics import seeds_summary

    seeds = [s for s in MULTI_SEEDS for _ in MULTI_LOADS][:nnets]
    loads = [L for _ in MULTI_SEEDS for L in MULTI_LOADS][:nnets]
    nets = [ax.Network(config_c(), device=dev) for _ in seeds]
    kw = dict(epochs=epochs, T=10, clamp_steps=5, stimcols=STIMCOLS, wave_t=35)
    try:
        res_p, rep_p = ax.multi_train(nets, seeds, loads, method="plain", **kw)
        res_m, rep_m = ax.multi_train(nets, seeds, loads, method="launch", autotune=True, graph=True, **kw)
    finally:
        for n in nets:
            n.close()
    assert res_m == res_p, "one-launch measurements differ from the plain path"
    rows = {L: printed(res_m[i]) for i, (s, L) in enumerate(zip(seeds, loads)) if s == 0}
    steps = rep_m["steps"]
    # algorithmic HBM bytes of the launch: W3 tiles read by the drive, branch updates of
    # the learning rule (4 planes read + written), conn and spikes per step, bias per
    # learning step
    alg = (1024.0 * rep_m["w3_tiles"] + 8192.0 * rep_m["learn_tasks"] + steps * (512 + 16) * 1024.0
           + rep_m["train_steps"] * 1024.0 * 1024.0)
    hbm_peak, pk = peaks()
    achieved = alg / (rep_m["gpu_ms"] / 1e3) / 1e9
    out = {"workload": f"{len(nets)} networks (seeds 0-4 x loads 12,24,36,48,60), config C, {epochs} epochs + readouts",
           "networks": len(nets), "network_steps": steps, "learning_steps": rep_m["train_steps"],
           "one_launch_ms": rep_m["gpu_ms"], "plain_ms": rep_p["gpu_ms"],
           "one_launch_steps_per_s": steps / (rep_m["gpu_ms"] / 1e3),
           "plain_steps_per_s": steps / (rep_p["gpu_ms"] / 1e3), "speedup_vs_plain": rep_p["gpu_ms"] / rep_m["gpu_ms"],
           "shape": {k: rep_m[k] for k in ("slots", "threads", "tiles", "grid", "graph", "tried")},
           "tune_ms": rep_m["tune_ms"], "bit_exact_vs_plain": True,
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
                        "peak_kind": pk, "w3_tiles": rep_m["w3_tiles"], "learn_tasks": rep_m["learn_tasks"],
                        "note": "algorithmic bytes = 1 KiB per W3 tile read + 8 KiB per learning branch update + "
                                "conn/spikes per step + bias per learning step"},
           "seed0_rows": rows}
    if epochs != EPOCHS or nnets != 25 or not pins:
        return out
    eq = table1_equal(rows)
    out["seed0_rows_equal_published_table1"] = all(eq.values())
    # Table 2: five-seed summaries; load 42 from five more networks
    per = {L: [printed(res_m[i]) for i, (s, LL) in enumerate(zip(seeds, loads)) if LL == L] for L in MULTI_LOADS}
    nets = [ax.Network(config_c(), device=dev) for _ in MULTI_SEEDS]
    try:
        r42, _ = ax.multi_train(nets, list(MULTI_SEEDS), [42] * 5, method="plain", **kw)
    finally:
        for n in nets:
            n.close()
    per[42] = [printed(r) for r in r42]
    summ = {str(L): seeds_summary(v) for L, v in sorted(per.items())}
    t2 = {str(r["stim"]): r for r in published()["table2"]["rows"]}
    fields = ("sustained_mean", "sustained_sd", "margin_mean", "margin_sd", "within_mean", "within_sd")
    out["table2"] = {"summary": summ, "equal_published": {L: all(summ[L][f] == t2[L][f] for f in fields) for L in t2}}
    out["table2"]["stim12_sustained_mean_equal_published"] = summ["12"]["sustained_mean"] == published()["table2"][
        "stim12_sustained_mean"]
    out["seed_means_equal_table2"] = all(out["table2"]["equal_published"].values())
    # Table 1 at the higher loads, seed 0
    hi = {}
    for method, lds in (("launch", [140, 200]), ("plain", [74, 90, 300])):
        nets = [ax.Network(config_c(), device=dev) for _ in lds]
        try:
            r, rep = ax.multi_train(nets, [0] * len(lds), lds, method=method, autotune=method == "launch", **kw)
        finally:
            for n in nets:
                n.close()
        hi.update({L: printed(x) for L, x in zip(lds, r)})
    out["table1_high_loads"] = {"rows": {str(L): hi[L] for L in sorted(hi)}, "equal_published": table1_equal(hi),
                                "methods": {"one launch": [140, 200], "plain": [74, 90, 300]}}
    return out


SERVE_LOADS = (12, 36, 60, 100, 140, 170, 200, 200)
SERVE_RATES = (2000, 10000, 50000)
SERVE_SECONDS = 1.0
SERVE_CHECK = {2000: None, 10000: 1000, 50000: 1000}  # requests checked against a plain recall (None = all)


def bench_serve(dev: int, rates=SERVE_RATES, seconds: float = SERVE_SECONDS, nnets: int = len(SERVE_LOADS)) -> dict:
    """Recall serving: 8 trained networks (config C, loads 12..200, seeds 0-7) answer
    Poisson-arriving recall requests (cue = 16-64 of a stored pattern's columns, 5 clamped
    + 10-60 free steps) with continuous batching; latency = result on the host - arrival.
    After each rate's run (outside its timed window) every request at 2,000 req/s, and
    1,000 spread over the others, are recomputed one at a time through the plain path and
    compared with the server's result."""
    import axon_b200 as ax

    loads = list(SERVE_LOADS[:nnets])
    seeds = list(range(len(loads)))
    nets = [ax.Network(config_c(), device=dev) for _ in seeds]
    try:
        _, rep = ax.multi_train(nets, seeds, loads, epochs=EPOCHS, T=10, clamp_steps=5, stimcols=STIMCOLS,
                                readout=False, autotune=True)
        pats = [ax.stimuli(sd, L, INCOLS, STIMCOLS) for sd, L in zip(seeds, loads)]
        refs = []  # clamped reference assemblies (active recurrent columns per pattern)
        for net, P in zip(nets, pats):
            cues = np.stack([ax.load_stim(P[q], 1.0, 2000 + q, NCOL) for q in range(len(P))])
            fin = net.recall(cues, 10, 10)["final"]
            refs.append([set(np.nonzero(fin[q, INCOLS:])[0].tolist()) for q in range(len(P))])
        out = {"workload": f"{len(nets)} networks (config C, loads {','.join(map(str, loads))}, seeds 0-{len(nets) - 1}); "
                           "Poisson arrivals; cue 16-64 columns of a stored pattern; 5 clamped + 10-60 free steps",
               "train_ms": rep["gpu_ms"], "rates": []}
        rng = np.random.default_rng(12345)
        tag = 0
        for rate in rates:
            srv = ax.Server(nets, 1 << 30)
            try:
                out["slots"] = srv.stats()["slots"]
                n = int(rate * seconds)
                gaps = rng.exponential(1.0 / rate, n)
                reqs = []
                for i in range(n):
                    net = int(rng.integers(len(nets)))
                    q = int(rng.integers(len(pats[net])))
                    size = int(rng.integers(16, 65))
                    cols = np.sort(rng.choice(pats[net][q], size, replace=False)).astype(np.uint32)
                    reqs.append((tag + i, net, q, cols, int(rng.integers(10, 61))))
                t0 = ax.clock_s() + 0.3
                arrive = t0 + np.cumsum(gaps)
                for (tg, net, q, cols, free), a in zip(reqs, arrive):
                    srv.submit(net, cols, 5, free, tg, float(a))
                lat, ov, last, got = [], [], 0.0, 0
                info = {r[0]: r for r in reqs}
                results = {}
                while got < n:
                    done = srv.poll(4096)
                    if not done:
                        time.sleep(0.002)
                        continue
                    for res, spk in done:
                        _, net, q, cols, free = info[res["tag"]]
                        lat.append(res["done_s"] - res["arrive_s"])
                        last = max(last, res["done_s"])
                        act = set(np.nonzero(spk[INCOLS:])[0].tolist())
                        ref = refs[net][q]
                        ov.append(len(act & ref) / np.sqrt(len(act) * len(ref)) if act and ref else 0.0)
                        results[res["tag"]] = spk
                    got += len(done)
                st = srv.stats()
            finally:
                srv.close()
            # after the timed window: each checked request alone through the plain path (64
            # steps at most, the length its per-step records hold), longer ones through a
            # batched recall of that one trajectory
            ncheck = n if SERVE_CHECK.get(rate) is None else min(n, SERVE_CHECK[rate])
            checked = reqs[:: max(1, n // ncheck)][:ncheck]
            mism = nplain = 0
            for tg, net, q, cols, free in checked:
                method = "plain" if 5 + free <= 64 else "batched"
                nplain += method == "plain"
                alone = nets[net].recall(ax.clamp_words(cols, NCOL)[None, :], 5 + free, 5, method=method)["final"][0]
                mism += int(not np.array_equal(alone, results[tg]))
            lat_ms = np.array(lat) * 1e3
            out["rates"].append({"offered_req_s": rate, "requests": n,
                                 "trajectories_per_s": n / (last - float(arrive[0])),
                                 "p50_ms": float(np.percentile(lat_ms, 50)), "p99_ms": float(np.percentile(lat_ms, 99)),
                                 "mean_overlap_with_reference": float(np.mean(ov)),
                                 "checked": len(checked), "checked_plain": nplain, "mismatches": mism,
                                 "mean_batch": st["mean_batch"], "max_batch": st["max_batch"]})
            tag += n
    finally:
        for x in nets:
            x.close()
    return out


def plain_alg_bytes(hist: np.ndarray, conn: np.ndarray) -> float:
    """Algorithmic HBM bytes of the plain path over the recorded trajectories: per
    trajectory-step 1 KiB per (column, branch) whose presynaptic group spiked at t-1
    (the W3 tiles k_drive must read), plus conn (512 KiB) and the spike vector (16 KiB)."""
    ngrp = NCOL // 8
    fan = np.bincount(conn.astype(np.int64), minlength=ngrp).astype(np.float64)
    act = (hist.reshape(hist.shape[0], hist.shape[1], ngrp, 8) != 0).any(-1)  # group spiked at t
    tiles = np.zeros(hist.shape[:2])
    tiles[:, 1:] = (act[:, :-1] * fan).sum(-1)
    return float((1024.0 * tiles + 512 * 1024 + 16 * 1024).sum())


def contraction_popcounts(hist: np.ndarray, conn: np.ndarray) -> float:
    """The AND-popcounts the batched contraction cannot avoid: per trajectory-step, for every
    (column, branch) whose presynaptic group spiked at t-1, one 32-bit AND-popcount per row
    (32 rows) and per nonzero spike word of the group."""
    ngrp = NCOL // 8
    fan = np.bincount(conn.astype(np.int64), minlength=ngrp).astype(np.float64)
    nzw = (hist.reshape(hist.shape[0], hist.shape[1], ngrp, 8) != 0).sum(-1)  # nonzero words per group
    return float(32.0 * (nzw[:, :-1] * fan).sum())


def cli_args() -> list[str]:
    return [f"{k}={v}" for k, v in CONFIG_C_KEYS.items()] + ["stimcols=64", "T=10", "clampsteps=5"]


def plain_train(dev: int, threads: int) -> dict:
    """The reference's one published throughput, config C timesteps/s while training
    (paper/axon_preprint.tex:667-669: 2,554-2,956 on an M1 Pro), measured as the reference
    measures it: the drop-in command line at loads 12-60, 40 epochs, seed 0, printing its
    'ms/timestep -> N steps/s' line and the five measurements (compared with Table 1).
    Beside it, the CPU oracle's training steps/s on the host cores over one epoch of
    load 12 (a bounded sample of the same presentations)."""
    from axon_b200 import build
    from tests.metrics import scrape

    exe = build.build_cli()
    rows = {}
    for L in MULTI_LOADS:
        t0 = time.time()
        p = subprocess.run([str(exe), *cli_args(), f"stim={L}", "epochs=40", "seed=0", "deep=1", "wave=1", "wavet=35",
                            f"device={dev}"], capture_output=True, text=True, timeout=900)
        if p.returncode != 0:
            raise RuntimeError(p.stderr)
        m = scrape(p.stdout)
        rows[L] = {"steps_per_s": float(m["steps_per_s"]), "wall_s": round(time.time() - t0, 2),
                   "within": f"{float(m['within_pct']):.2f}", "recall": m["recall"], "best_other": m["best_other"],
                   "margin": m["margin"], "sustained": m["sustained"], "drive": m["drive_t6"]}
    eq = table1_equal({L: r for L, r in rows.items()})
    # CPU oracle: one epoch of load-12 learning presentations on the host cores
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_lib as O

    cpu = O.OracleNet(O.config(ncol=NCOL, incols=INCOLS, **CONFIG_C_KEYS), threads=threads)
    cpu.init(SEED)
    pats = O.stimuli(SEED, 12, INCOLS, STIMCOLS)
    t0 = time.perf_counter()
    for p in range(12):
        cpu.present(O.load_stim(pats[p], 1.0, 1000 + p, NCOL), 10, 5, True)
    cpu_s = time.perf_counter() - t0
    cpu.close()
    return {"workload": "config C training, 40 epochs, seed 0, through the axon command line (drop-in)",
            "steps_per_s": {str(L): r["steps_per_s"] for L, r in rows.items()}, "rows": {str(L): r for L, r in rows.items()},
            "rows_equal_table1": eq,
            "published_m1_pro_steps_per_s": "2554-2956 (paper/axon_preprint.tex:667-669; context only, not on this box)",
            "cpu_oracle": {"steps_per_s": 120 / cpu_s, "cores": threads,
                           "sample": "1 epoch of load 12 (12 learning presentations x 10 steps)"}}


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons while running."""

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "25"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.rows.append([x.strip() for x in ln.split(",")])

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            self.proc.wait(timeout=5)

    def summary(self) -> dict:
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 2 + i and r[2 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def measured_traffic(kernel: str):
    """DRAM bytes per launch of `kernel` from its committed ncu capture (profiles/), or None."""
    p = ROOT / "profiles" / "traffic.json"
    if not p.exists():
        return None
    return json.loads(p.read_text()).get(kernel, {}).get("dram_bytes_per_launch")


def peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def cpu_sample(gpu_net, cues, ev, gpu_hist, threads: int, ntraj: int) -> dict:
    """The CPU oracle on a bounded sample of the same trajectories (same trained state),
    timed, and each sampled trajectory compared with the GPU's spike history."""
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_lib as O

    cpu = O.OracleNet(O.config(ncol=NCOL, incols=INCOLS, **CONFIG_C_KEYS), threads=threads)
    for name in ("W0", "W1", "W2", "W3", "CONN", "BIAS"):
        cpu.write(name, gpu_net.read(name))
    idx = np.linspace(0, cues.shape[0] - 1, ntraj).astype(int)
    dt, mism = 0.0, 0
    for b in idx:
        t0 = time.perf_counter()
        cpu.present(cues[b], T_RECALL, CLAMP_RECALL, False, True, 0)
        dt += time.perf_counter() - t0
        h = cpu.read("HIST")[: T_RECALL * NCOL].reshape(T_RECALL, NCOL)
        mism += int(not np.array_equal(h, gpu_hist[b]))
    cpu.close()
    return {"value": float(ev[idx].sum() / dt), "unit": "synaptic events/s", "cores": threads, "kind": "port",
            "sample": f"{ntraj} of the 300 trajectories (evenly spread over clean and noisy cues) x {T_RECALL} steps, "
                      f"oracle present(learn=0), {dt:.1f} s",
            "oracle_match": {"checked": int(ntraj), "mismatches": mism, "compared": "full spike history vs the GPU's"}}


def run_reference(args) -> None:
    """Reference arm: the CPU restatement of the reference (oracle) on the host cores. It
    loads nothing from the engine: configuration, patterns and cues come from the oracle
    library alone. Its trained planes and its sampled trajectories are checked against the
    oracle fixture of this workload, the same fixture the GPU arm is checked against."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_lib as O

    threads = os.cpu_count() or 1
    cfg = O.config(ncol=NCOL, incols=INCOLS, **CONFIG_C_KEYS)
    pats = O.stimuli(SEED, LOAD, INCOLS, STIMCOLS)
    cues = make_cues(pats, O.noisy_cue, O.noisy_seed)
    cpu = O.OracleNet(cfg, threads=threads)
    cpu.init(SEED)
    train_s = train(cpu, pats, O.load_stim)
    fx = fixture()
    planes_ok = fx is not None and trained_digest(cpu) == fx["trained_sha256_w0_w3_bias"]
    conn = cpu.read("CONN")
    ntraj = max(1, args.ref_traj)
    idx = np.linspace(0, cues.shape[0] - 1, ntraj).astype(int)
    times, evs = [], []
    hists = []
    for it in range(args.warmup + args.steps):
        t1 = time.perf_counter()
        hists = []
        for b in idx:
            cpu.present(cues[b], T_RECALL, CLAMP_RECALL, False, True, 0)
            hists.append(cpu.read("HIST")[: T_RECALL * NCOL].reshape(T_RECALL, NCOL))
        dt = time.perf_counter() - t1
        ev = events_per_step(np.stack(hists), conn).sum()
        if it >= args.warmup:
            times.append(dt)
            evs.append(ev)
    match = check_against_fixture(fx, idx, hists)
    cpu.close()
    value = float(sum(evs) / sum(times))
    line = {"impl": "reference", "metric": "synaptic events/s (batched recall, 300 trajectories x 45 steps)",
            "value": value, "unit": "synaptic events/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded cues)",
            "config": {"workload": "batched recall, config C load 60 seed 0, 300 cues (whole patterns and 10 %/25 % "
                                   "active bits flipped) x (10 clamp + 35 free)",
                       "sample_trajectories": int(ntraj), "train_s": round(train_s, 1)},
            "trained_planes_equal_oracle_fixture": planes_ok, "oracle_match": match,
            "cpu_baseline": {"value": value, "unit": "synaptic events/s", "cores": threads, "kind": "port",
                             "sample": f"{ntraj} of the 300 trajectories (evenly spread) x {T_RECALL} steps per step"},
            "e2e": {"value": value, "unit": "synaptic events/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def time_device(net, d_cues, B, T, clamp, d_final, flush, steps, contraction="popc", slab="floor") -> list[float]:
    import torch

    times = []
    for _ in range(steps):
        flush.zero_()  # evict L2 between timed steps (untimed: outside the device-timed launch)
        torch.cuda.synchronize()
        times.append(net.recall_device(d_cues.data_ptr(), B, T, clamp, d_final.data_ptr(), graph=True,
                                       contraction=contraction, slab=slab))
    torch.cuda.synchronize()
    return times


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="axon", choices=["axon", "reference"])
    ap.add_argument("--ref-traj", type=int, default=30)
    ap.add_argument("--cpu-traj", type=int, default=120)
    ap.add_argument("--contraction", default="popc", choices=["popc", "tensor"],
                    help="AND-popcount unit of the timed batched recall (the other one is timed in the A/B block)")
    ap.add_argument("--no-ab", action="store_true", help="skip the contraction A/B and the wave variant")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain-path comparison")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end (host buffer) measurement")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU oracle sample")
    ap.add_argument("--no-multi", action="store_true", help="skip the 25-network one-launch measurement")
    ap.add_argument("--no-pins", action="store_true", help="skip the Table 2 / high-load Table 1 networks")
    ap.add_argument("--no-serve", action="store_true", help="skip the recall-serving measurement")
    ap.add_argument("--no-train", action="store_true", help="skip the command-line training throughput")
    ap.add_argument("--multi-nets", type=int, default=25, help="networks of the multi-network block (small cases)")
    ap.add_argument("--multi-epochs", type=int, default=EPOCHS)
    ap.add_argument("--serve-rates", default=",".join(map(str, SERVE_RATES)), help="offered loads, requests/s")
    ap.add_argument("--serve-seconds", type=float, default=SERVE_SECONDS)
    ap.add_argument("--serve-nets", type=int, default=len(SERVE_LOADS))
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
        return
    assert args.warmup >= 3, "at least 3 warm-up steps"
    from axon_b200.replicas import Replicas

    rep = Replicas.from_env(args.gpus)
    rank, world = rep.rank, rep.world
    import torch

    import axon_b200 as ax
    from axon_b200 import build

    if rank == 0:
        build.build_lib()
        build.build_cli()
    rep.barrier()
    dev = torch.cuda.current_device()
    net = ax.Network(config_c(), device=dev)
    net.init(SEED)
    pats = ax.stimuli(SEED, LOAD, INCOLS, STIMCOLS)
    train_s = train(net, pats, ax.load_stim)
    fx = fixture()
    planes_ok = fx is not None and trained_digest(net) == fx["trained_sha256_w0_w3_bias"]
    cues = make_cues(pats, ax.noisy_cue, ax.noisy_cue_seed)
    B = cues.shape[0]
    # events of the workload (fixed by the trajectories), from one recorded run, and every
    # trajectory against the oracle's fixture
    ctr = args.contraction
    ref = net.recall(cues, T_RECALL, CLAMP_RECALL, hist=True, contraction=ctr)
    conn = net.read("CONN")
    ev = events_per_step(ref["hist"], conn)
    events = float(ev.sum())
    match = check_against_fixture(fx, range(B), ref["hist"])
    match["trained_planes_equal"] = planes_ok

    # device-resident inputs and outputs
    d_cues = torch.from_numpy(cues.view(np.int32)).to(f"cuda:{dev}")
    d_final = torch.empty((B, NCOL), dtype=torch.int32, device=f"cuda:{dev}")
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.int32, device=f"cuda:{dev}")
    for _ in range(args.warmup):  # the first call captures the launch as a CUDA graph, the rest replay it
        net.recall_device(d_cues.data_ptr(), B, T_RECALL, CLAMP_RECALL, d_final.data_ptr(), graph=True, contraction=ctr)
    assert np.array_equal(d_final.cpu().numpy().view(np.uint32), ref["final"])
    torch.cuda.synchronize()
    rep.barrier()
    with ClockSampler(dev) as clk:
        times = time_device(net, d_cues, B, T_RECALL, CLAMP_RECALL, d_final, flush, args.steps, ctr)
    rep.barrier()
    ms = rep.max(float(np.mean(times)))
    value = world * events / (ms / 1e3)

    # end to end through the public C-ABI call with pinned host buffers
    h_cues = torch.from_numpy(cues.view(np.int32)).pin_memory().numpy().view(np.uint32)
    h_final = torch.empty(cues.shape, dtype=torch.int32).pin_memory().numpy().view(np.uint32)
    e2e_t = []
    for it in range(0 if args.no_e2e else args.warmup + max(3, args.steps // 2)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = net.recall(h_cues, T_RECALL, CLAMP_RECALL, graph=True, final_out=h_final, contraction=ctr)
        dt = time.perf_counter() - t0
        if it >= args.warmup:
            e2e_t.append(dt)
    if e2e_t:
        assert np.array_equal(r["final"], ref["final"])
    e2e_s = rep.max(float(np.mean(e2e_t)) if e2e_t else float("nan"))

    wave = contraction = slab = None
    if not args.no_ab:
        # the reference-parity variant: the wave readout's 5 clamped + 30 free steps
        rw = net.recall(cues, T_WAVE, CLAMP_WAVE, hist=True, contraction=ctr)
        ev_w = float(events_per_step(rw["hist"], conn).sum())
        d_fw = torch.empty((B, NCOL), dtype=torch.int32, device=f"cuda:{dev}")
        for _ in range(args.warmup):
            net.recall_device(d_cues.data_ptr(), B, T_WAVE, CLAMP_WAVE, d_fw.data_ptr(), graph=True, contraction=ctr)
        assert np.array_equal(d_fw.cpu().numpy().view(np.uint32), rw["final"])
        tw = time_device(net, d_cues, B, T_WAVE, CLAMP_WAVE, d_fw, flush, max(5, args.steps // 2), ctr)
        ms_w = rep.max(float(np.mean(tw)))
        wave = {"workload": "the same 300 cues x (5 clamp + 30 free), the reference's wave readout "
                            "(src/axon.mm:1804-1858)",
                "value": world * ev_w / (ms_w / 1e3), "unit": "synaptic events/s", "ms_per_step": ms_w,
                "events_per_batch": ev_w}
        # A/B of the contraction unit: the same batch with k_drive's AND-popcounts on the other
        # unit (tensor cores: binary MMA m16n8k256 and.popc; CUDA cores: __popc)
        other = "tensor" if ctr == "popc" else "popc"
        ro = net.recall(cues, T_RECALL, CLAMP_RECALL, hist=True, contraction=other)
        other_exact = bool(np.array_equal(ro["hist"], ref["hist"]))
        for _ in range(args.warmup):
            net.recall_device(d_cues.data_ptr(), B, T_RECALL, CLAMP_RECALL, d_fw.data_ptr(), graph=True,
                              contraction=other)
        to = time_device(net, d_cues, B, T_RECALL, CLAMP_RECALL, d_fw, flush, max(5, args.steps // 2), other)
        ms_o = rep.max(float(np.mean(to)))
        per = {ctr: ms, other: ms_o}
        contraction = {"popc_ms_per_step": per["popc"], "tensor_ms_per_step": per["tensor"],
                       "timed_as_value": ctr, f"{other}_bit_exact": other_exact,
                       "faster": min(per, key=per.get),
                       "note": "tensor = mma.sync m16n8k256 b1 and.popc, 8 entries x 32 rows per chunk; popc = __popc "
                               "on the CUDA cores"}
        # A/B of the drive slab: every per-neuron drive stored (full) against only those at or
        # above each trajectory's histogram floor (the default)
        rf = net.recall(cues, T_RECALL, CLAMP_RECALL, hist=True, contraction=ctr, slab="full")
        full_exact = bool(np.array_equal(rf["hist"], ref["hist"]))
        for _ in range(args.warmup):
            net.recall_device(d_cues.data_ptr(), B, T_RECALL, CLAMP_RECALL, d_fw.data_ptr(), graph=True,
                              contraction=ctr, slab="full")
        tf = time_device(net, d_cues, B, T_RECALL, CLAMP_RECALL, d_fw, flush, max(5, args.steps // 2), ctr, "full")
        slab = {"floor_ms_per_step": ms, "full_ms_per_step": rep.max(float(np.mean(tf))), "full_bit_exact": full_exact,
                "note": "floor = per-neuron drives stored for columns at or above the trajectory's histogram floor "
                        "(all at the step after the clamp; gated columns without one recomputed); full = all stored"}

    # plain GPU path on the same 300 trajectories (one persistent launch per trajectory)
    plain = None
    hbm_peak, pk = peaks()
    if not args.no_plain:
        rp = net.recall(cues, T_RECALL, CLAMP_RECALL, method="plain")
        assert np.array_equal(rp["final"], ref["final"])
        pt = [net.recall_device(d_cues.data_ptr(), B, T_RECALL, CLAMP_RECALL, d_final.data_ptr(), method="plain")
              for _ in range(2)]
        pms = rep.max(float(np.mean(pt)))
        pa = plain_alg_bytes(ref["hist"], conn) / (pms / 1e3) / 1e9
        plain = {"value": world * events / (pms / 1e3), "ms_per_step": pms, "launches_per_step": B,
                 "us_per_trajectory_step": 1e3 * pms / (B * T_RECALL),
                 "roofline": {"bound": "hbm", "achieved": pa, "peak": hbm_peak, "unit": "GB/s", "frac": pa / hbm_peak,
                              "peak_kind": pk, "note": "algorithmic bytes = sum over trajectory-steps of 1 KiB per "
                                                       "(column, branch) with a spiking group + conn + spikes"}}

    threads = os.cpu_count() or 1
    ptrain = None if (args.no_train or rank != 0 or world != 1) else plain_train(dev, threads)
    multi = None if args.no_multi else bench_multi(dev, args.multi_nets, args.multi_epochs, not args.no_pins)
    serving = None if args.no_serve else bench_serve(dev, [int(x) for x in args.serve_rates.split(",")],
                                                     args.serve_seconds, args.serve_nets)

    if rank != 0:
        rep.close()
        return
    # roofline of the batched kernel, strict algorithmic bytes: W3 (128 MiB, read once per
    # recall step for all trajectories) + every trajectory's spike vector read and written
    # per step
    w3_bytes = NCOL * 32 * 1024
    spikes = 2 * B * NCOL * 4
    alg_bytes = T_RECALL * (w3_bytes + spikes)
    achieved = alg_bytes / (ms / 1e3) / 1e9
    pops = contraction_popcounts(ref["hist"], conn)
    sm_mhz = clk.summary().get("sm_mhz") or 1965.0
    peak_pops = torch.cuda.get_device_properties(dev).multi_processor_count * 16 * sm_mhz * 1e6
    cpu = None if (args.no_cpu or world != 1) else cpu_sample(net, cues, ev, ref["hist"], threads, args.cpu_traj)
    line = {
        "metric": "synaptic events/s (batched recall, 300 trajectories x 45 steps)",
        "value": value, "unit": "synaptic events/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic (seeded cues from the reference's stimulus stream)",
        "config": {"workload": "batched recall, config C load 60 seed 0, 300 cues (whole patterns, and 10 %/25 % of "
                               "their active bits flipped off, 2 draws each) x (10 clamp + 35 free), bias off",
                   "trajectories": B, "steps_per_trajectory": T_RECALL, "events_per_batch": events,
                   "train_s": round(train_s, 2), "l2": "flushed between timed steps (256 MiB write)",
                   "launch": "one persistent cooperative kernel per batch, replayed as a captured CUDA graph",
                   "parallelism": f"replicas x{world}"},
        "oracle_match": match,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
                     "traffic": measured_traffic("k_recall"), "peak_kind": pk,
                     "note": "algorithmic bytes = 45 x (W3 128 MiB + every trajectory's spike vector in and out); "
                             "the kernel is bound by the popcount (XU) pipe and issue, see profiles/"},
        "int_roofline": {"bound": "xu (popcount pipe)", "achieved": pops / (ms / 1e3), "unit": "popcounts/s",
                         "peak": peak_pops, "frac": pops / (ms / 1e3) / peak_pops,
                         "note": "the contraction's unavoidable 32-bit AND-popcounts (32 rows x nonzero spike words "
                                 "of every active (column, branch, trajectory)) per second, against 16 popcounts per SM "
                                 "per clock at the sampled SM clock; ncu's XU-pipe utilisation is the same measure"},
        "cpu_baseline": cpu,
        "e2e": {"value": world * events / e2e_s, "unit": "synaptic events/s",
                "h2d_bytes_per_step": int(B * INCOLS * 4),  # the cues' input columns: all the clamp reads
                "d2h_bytes_per_step": int(B * NCOL * 4)},
        "wave_variant": wave,
        "contraction_ab": contraction,
        "slab_ab": slab,
        "plain": plain,
        "batched_over_plain": (value / plain["value"]) if plain else None,
        "plain_train": ptrain,
        "multi": multi,
        "serving": serving,
        "gpu_launches": args.steps,
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)
    rep.close()


if __name__ == "__main__":
    main()
