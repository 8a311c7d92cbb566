"""The engine pinned to numbers the reference itself holds, beyond the spot-check row:

* the published capacity sweep (paper/axon_preprint.tex:262-272, bench/cap10.sh) at the
  loads the serving and scaling workloads train (74, 90, 140, 200, 300; seed 0), through
  the one-launch multi-network path (140, 200: the path the serving networks are trained
  with) and the plain path;
* the published five-seed replication (paper/axon_preprint.tex:288-292, bench/seeds.sh):
  means and sample standard deviations of the sustained ratio, margin and within-assembly
  density over seeds 0-4 at loads 24, 36, 42, 48, 60, and the 12-pattern sustained mean
  of the text (tex:298-299);
* the batched-recall benchmark workload (config C, load 60, 300 cues of 45 steps) against
  the CPU oracle's recorded answer, tests/golden/recall_load60.json: the trained planes and
  every trajectory's spike history.
"""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

from metrics import seeds_summary

pytestmark = pytest.mark.gpu

GOLD = json.loads((Path(__file__).parent / "golden" / "published.json").read_text())
RECALL = Path(__file__).parent / "golden" / "recall_load60.json"
KW = dict(epochs=40, T=10, clamp_steps=5, stimcols=64, wave_t=35)


def cfg_c():
    import axon_b200 as ax

    return ax.config(ncol=4096, incols=512, **ax.CONFIG_C)


def printed(r: dict) -> dict:
    first, last = float(f"{r['wave_first']:.3f}"), float(f"{r['wave_last']:.3f}")
    return {"within": f"{r['within_pct']:.2f}", "within_pct": f"{r['within_pct']:.4f}", "recall": f"{r['recall']:.3f}",
            "best_other": f"{r['best_other']:.3f}", "margin": f"{r['recall'] - r['best_other']:+.3f}",
            "sustained": f"{last / first:.3f}", "drive": f"{r['drive_t6']:.0f}"}


def train_fleet(seeds, loads, method):
    import axon_b200 as ax

    nets = [ax.Network(cfg_c()) for _ in seeds]
    try:
        res, _ = ax.multi_train(nets, list(seeds), list(loads), method=method, autotune=method == "launch", **KW)
    finally:
        for n in nets:
            n.close()
    return [printed(r) for r in res]


@pytest.mark.parametrize("method,loads", [("launch", (140, 200)), ("plain", (74, 90, 300))])
def test_table1_high_loads(method, loads):
    gold = {r["stim"]: r for r in GOLD["table1"]}
    for L, m in zip(loads, train_fleet([0] * len(loads), loads, method)):
        exp = gold[L]
        got = {k: m[k] for k in ("within", "recall", "best_other", "margin", "sustained", "drive")}
        assert got == {k: exp[k] for k in got}, f"load {L}"


def test_table2_five_seed_replication():
    t2 = GOLD["table2"]
    loads = [12, 24, 36, 42, 48, 60]
    seeds = [s for s in t2["seeds"] for _ in loads]
    lds = [L for _ in t2["seeds"] for L in loads]
    rows = train_fleet(seeds, lds, "plain")
    for L in loads:
        summ = seeds_summary([m for m, LL in zip(rows, lds) if LL == L])
        if L == 12:
            assert summ["sustained_mean"] == t2["stim12_sustained_mean"]
            continue
        exp = next(r for r in t2["rows"] if r["stim"] == L)
        for f in ("sustained_mean", "sustained_sd", "margin_mean", "margin_sd", "within_mean", "within_sd"):
            assert summ[f] == exp[f], f"load {L} {f}: {summ[f]} vs published {exp[f]}"


@pytest.mark.skipif(not RECALL.exists(), reason="oracle fixture tests/golden/recall_load60.json not generated")
def test_benchmark_workload_matches_oracle_fixture():
    import axon_b200 as ax

    fx = json.loads(RECALL.read_text())
    digest = lambda *a, n=None: (lambda h: h[:n] if n else h)(  # noqa: E731
        hashlib.sha256(b"".join(np.ascontiguousarray(x, dtype="<u4").tobytes() for x in a)).hexdigest())
    net = ax.Network(cfg_c())
    net.init(fx["seed"])
    pats = ax.stimuli(fx["seed"], fx["load"], 512, 64)
    for _ in range(fx["epochs"]):
        for p in range(fx["load"]):
            net.present(ax.load_stim(pats[p], 1.0, 1000 + p, 4096), 10, 5, True)
    net.present(ax.load_stim(pats[0], 1.0, 31337, 4096), 10, 5, True)
    assert digest(*(net.read(n) for n in ("W0", "W1", "W2", "W3", "BIAS"))) == fx["trained_sha256_w0_w3_bias"]
    cues = [ax.noisy_cue(pats[q], 0.0, 0, 4096) for q in range(fx["load"])]
    for pct in fx["flip_pcts"]:
        for d in range(fx["draws"]):
            cues += [ax.noisy_cue(pats[q], pct / 100, ax.noisy_cue_seed(q, pct, d), 4096) for q in range(fx["load"])]
    out = net.recall(np.stack(cues), fx["T"], fx["clamp_steps"], hist=True)
    bad = [b for b, row in enumerate(fx["trajectories"])
           if digest(out["hist"][b], n=16) != row["hist"] or digest(out["final"][b], n=16) != row["final"]]
    net.close()
    assert not bad, f"{len(bad)} of {len(cues)} trajectories differ from the oracle, first {bad[:5]}"
