"""Many networks of uneven load in one persistent launch (axon_multi_train).

Parity chain: the one-launch form leaves every network's weights, bias and measurements
exactly as the plain path does (one presentation launch at a time, the same program);
every fixed launch shape agrees with the autotuned one; and each network's measurements
equal what the `axon` command line (itself line-for-line equal to the CPU oracle) prints
for that seed and load."""
import numpy as np
import pytest

import axon_b200 as ax
from metrics import scrape
from test_gpu_cli import CONFIG_C, engine_cli

pytestmark = pytest.mark.gpu

SMALL_ARGS = ["ncol=512", "incols=64", "stimcols=16", "target=24"]
SMALL_CFG = dict(ax.CONFIG_C, ncol=512, incols=64, target=24)
SEEDS = [0, 1, 2, 3, 4]
LOADS = [3, 5, 2, 6, 4]
EPOCHS = 2
PLANES = ("W0", "W1", "W2", "W3", "BIAS")


def train(method="launch", seeds=SEEDS, loads=LOADS, **kw):
    nets = [ax.Network(SMALL_CFG) for _ in seeds]
    try:
        res, rep = ax.multi_train(nets, seeds, loads, epochs=EPOCHS, stimcols=16, method=method, **kw)
        state = [{b: n.read(b) for b in PLANES} for n in nets]
    finally:
        for n in nets:
            n.close()
    return res, rep, state


def printed(r: dict) -> dict:
    """The measurements as the command line prints them (and bench/cap10.sh scrapes them)."""
    first, last = float(f"{r['wave_first']:.3f}"), float(f"{r['wave_last']:.3f}")
    return {"within_pct": f"{r['within_pct']:.4f}", "recall": f"{r['recall']:.3f}",
            "best_other": f"{r['best_other']:.3f}", "margin": f"{r['recall'] - r['best_other']:+.3f}",
            "drive_t6": f"{r['drive_t6']:.0f}", "sustained": f"{last / first:.3f}"}


@pytest.fixture(scope="module")
def plain():
    return train("plain")


def assert_same(a, b):
    res_a, _, st_a = a
    res_b, _, st_b = b
    assert res_a == res_b
    for x, y in zip(st_a, st_b):
        for name in PLANES:
            assert np.array_equal(x[name], y[name]), name


def test_one_launch_equals_plain_path(plain):
    got = train("launch", autotune=True, graph=True)
    rep = got[1]
    assert rep["graph"] == 1 and rep["tried"] > 0 and rep["slots"] >= 1
    assert rep["steps"] == plain[1]["steps"] == sum(r["steps"] for r in got[0])
    assert_same(got, plain)


@pytest.mark.parametrize("slots,threads", [(1, 1024), (2, 512), (5, 1024), (3, 512), (4, 1024), (3, 896), (5, 896)])
def test_every_shape_gives_the_same_networks(plain, slots, threads):
    got = train("launch", autotune=False, slots=slots, threads=threads, graph=False)
    assert got[1]["slots"] == slots and got[1]["threads"] == threads
    assert_same(got, plain)


def test_measurements_match_command_line(plain):
    res = plain[0]
    for i, (seed, load) in enumerate(zip(SEEDS, LOADS)):
        out = engine_cli([*CONFIG_C, *SMALL_ARGS, f"stim={load}", f"seed={seed}", f"epochs={EPOCHS}", "deep=1",
                          "wave=1", "wavet=35"])
        m = scrape(out)
        want = {k: m[k] for k in ("within_pct", "recall", "best_other", "margin", "drive_t6", "sustained")}
        assert printed(res[i]) == want, (seed, load)


def test_training_only_and_bad_arguments():
    res, rep, _ = train("launch", readout=False, autotune=False, slots=2)
    assert all(r["within_pct"] == 0.0 for r in res)
    assert rep["steps"] == rep["train_steps"] == sum((EPOCHS * L + 1) * 10 for L in LOADS)
    nets = [ax.Network(SMALL_CFG) for _ in range(2)]
    try:
        with pytest.raises(ax._capi.AxonError):
            ax.multi_train([nets[0], nets[0]], [0, 1], [2, 2], epochs=1, stimcols=16)  # same network twice
        with pytest.raises(ax._capi.AxonError):
            ax.multi_train(nets, [0, 1], [2, 0], epochs=1, stimcols=16)  # empty load
    finally:
        for n in nets:
            n.close()


@pytest.mark.parametrize("variant", [dict(margingate=1, hetero=1, ltdrep=2, ltdevery=1), dict(contrast=0),
                                     dict(mode=0, dthr=2), dict(mode=2, dthr=3, boost=7), dict(topkpar=0),
                                     dict(biasdownevery=3, biasshift=2, ktest=8, facil=5)])
def test_rule_variants_one_launch_equals_plain(variant):
    """Learning-rule and mode variants: the one-launch form leaves the same weights, bias
    and measurements as the plain path."""
    cfg = dict(SMALL_CFG, **variant)

    def run(method, **kw):
        nets = [ax.Network(cfg) for _ in range(3)]
        try:
            res, _ = ax.multi_train(nets, [0, 1, 2], [3, 4, 2], epochs=2, stimcols=16, method=method, **kw)
            return res, [{b: n.read(b) for b in PLANES} for n in nets]
        finally:
            for n in nets:
                n.close()

    a = run("launch", autotune=False, slots=3, threads=512, graph=False)
    b = run("plain")
    assert a[0] == b[0]
    for x, y in zip(a[1], b[1]):
        for name in PLANES:
            assert np.array_equal(x[name], y[name]), (variant, name)
