"""Regenerates tests/golden/recall_load60.json: the CPU oracle's answer for the
batched-recall workload, so that the engine's results on it (and the CPU reference arm's)
can be checked against the oracle without rerunning it.

Workload: config C (ncol 4096, incols 512), seed 0, 60 patterns of 64 columns, trained
for 40 epochs as the reference's schedule does (every pattern once per epoch, seed
1000 + p, T = 10, 5 clamped steps, learning on; then one more learning presentation of
pattern 0, seed 31337). Then 300 readouts with the bias off, 10 clamped + 35 free steps:
the 60 whole patterns, then for each fraction (10 %, 25 %) and draw (0, 1) the 60
patterns with that fraction of their active bits flipped off (noisy cue, seed
90000 + 1000 * pct + 16 * q + draw).

Recorded: a SHA-256 of the trained W0..W3 and bias words, and for every trajectory the
first 16 hex digits of the SHA-256 of its final spike vector and of its whole spike
history (45 x 4096 words, little-endian), and its synaptic-event count.

    python tests/golden/make_recall_golden.py     # ~10 min on 8 cores
"""
from __future__ import annotations

import hashlib
import json
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))

import oracle_lib as O  # noqa: E402

NCOL, INCOLS, STIMCOLS, LOAD, EPOCHS, SEED = 4096, 512, 64, 60, 40, 0
T_RECALL, CLAMP_RECALL = 45, 10
FLIP_PCTS, DRAWS = (10, 25), 2
CONFIG_C = dict(nand=4, target=64, k=24, dthr=1, mode=1, inbr=4, contrast=1, margingate=0, ltdrep=1, ltdevery=2,
                biasup=73, biasdown=1)


def digest(*arrays: np.ndarray, n: int | None = None) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a, dtype="<u4").tobytes())
    return h.hexdigest()[:n] if n else h.hexdigest()


def cue_list(pats: np.ndarray, noisy_cue, noisy_seed) -> list[tuple[str, np.ndarray]]:
    """The 300 cues in batch order, each with its label (q, pct, draw)."""
    cues = [(f"q{q}", noisy_cue(pats[q], 0.0, 0, NCOL)) for q in range(LOAD)]
    for pct in FLIP_PCTS:
        for d in range(DRAWS):
            for q in range(LOAD):
                cues.append((f"q{q}_flip{pct}_d{d}", noisy_cue(pats[q], pct / 100.0, noisy_seed(q, pct, d), NCOL)))
    return cues


def events(hist: np.ndarray, conn: np.ndarray) -> int:
    """Synaptic events of one trajectory: per step t >= 1, 32 x the spikes at t-1 of each
    (column, branch)'s presynaptic group."""
    ngrp = NCOL // 8
    fan = np.bincount(conn.astype(np.int64), minlength=ngrp)
    pc = np.bitwise_count(hist).reshape(hist.shape[0], ngrp, 8).sum(-1, dtype=np.int64)
    return int(32 * (pc[:-1] * fan).sum())


def train(net, pats, load_stim) -> None:
    for _ in range(EPOCHS):
        for p in range(LOAD):
            net.present(load_stim(pats[p], 1.0, 1000 + p, NCOL), 10, 5, True)
    net.present(load_stim(pats[0], 1.0, 31337, NCOL), 10, 5, True)  # the reference's extra presentation


def main() -> None:
    cfg = O.config(ncol=NCOL, incols=INCOLS, **CONFIG_C)
    net = O.OracleNet(cfg, threads=O.default_threads())
    net.init(SEED)
    pats = O.stimuli(SEED, LOAD, INCOLS, STIMCOLS)
    t0 = time.time()
    train(net, pats, O.load_stim)
    train_s = time.time() - t0
    planes = digest(*(net.read(n) for n in ("W0", "W1", "W2", "W3", "BIAS")))
    conn = net.read("CONN")
    rows = []
    for label, cue in cue_list(pats, O.noisy_cue, O.noisy_seed):
        net.present(cue, T_RECALL, CLAMP_RECALL, False, True, 0)
        hist = net.read("HIST")[: T_RECALL * NCOL].reshape(T_RECALL, NCOL)
        rows.append({"cue": label, "final": digest(hist[-1], n=16), "hist": digest(hist, n=16),
                     "events": events(hist, conn)})
    net.close()
    fx = {"generator": "tests/golden/make_recall_golden.py", "oracle": "oracle/_build/liboracle.so",
          "config": {"ncol": NCOL, "incols": INCOLS, **CONFIG_C}, "load": LOAD, "seed": SEED, "epochs": EPOCHS,
          "T": T_RECALL, "clamp_steps": CLAMP_RECALL, "flip_pcts": list(FLIP_PCTS), "draws": DRAWS,
          "trained_sha256_w0_w3_bias": planes, "train_s": round(train_s, 1), "trajectories": rows}
    (HERE / "recall_load60.json").write_text(json.dumps(fx, indent=0) + "\n")
    print(f"trained in {train_s:.0f} s; {len(rows)} trajectories; planes {planes[:16]}")


if __name__ == "__main__":
    main()
