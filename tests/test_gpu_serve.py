"""Recall serving with continuous batching (axon_serve_*).

Each request is a readout trajectory: its cue columns clamped for the first steps, then
free steps (present() with learn = 0). The server advances all admitted trajectories
together, tick by tick, admitting new ones as slots free up; a network with many
trajectories in a tick is advanced by the batched drive kernel, one with few by the
gather kernel. The tests show that a request's final spikes are the same alone and in the
mix (all at once, staggered, and squeezed through a few slots), and the same as
axon_recall's for that network and cue."""
import numpy as np
import pytest

import axon_b200 as ax

pytestmark = pytest.mark.gpu

CFG = dict(ax.CONFIG_C, ncol=512, incols=64, target=24)
SEEDS, LOADS, STIMCOLS = [0, 1, 2], [3, 5, 4], 16
CLAMP = 5


@pytest.fixture(scope="module")
def fleet():
    nets = [ax.Network(CFG) for _ in SEEDS]
    ax.multi_train(nets, SEEDS, LOADS, epochs=2, stimcols=STIMCOLS, readout=False, autotune=False, slots=3)
    pats = [ax.stimuli(s, L, 64, STIMCOLS) for s, L in zip(SEEDS, LOADS)]
    yield nets, pats
    for n in nets:
        n.close()


def requests(pats, n, seed):
    rng = np.random.default_rng(seed)
    out = []
    for tag in range(n):
        net = int(rng.integers(len(pats)))
        q = int(rng.integers(len(pats[net])))
        size = int(rng.integers(2, STIMCOLS + 1))
        cols = np.sort(rng.choice(pats[net][q], size, replace=False)).astype(np.uint32)
        out.append(dict(tag=tag, net=net, cols=cols, free=int(rng.integers(3, 13))))
    return out


def serve(nets, reqs, mem_bytes=64 << 20, spread_s=0.0):
    got = {}
    with ax.Server(nets, mem_bytes) as srv:
        t0 = ax.clock_s()
        for i, r in enumerate(reqs):
            arrive = t0 + spread_s * i / max(1, len(reqs)) if spread_s else 0.0
            srv.submit(r["net"], r["cols"], CLAMP, r["free"], r["tag"], arrive)
        srv.wait_idle(120)
        for res, spk in srv.poll(len(reqs) + 8):
            got[res["tag"]] = (res, spk)
        st = srv.stats()
    assert len(got) == len(reqs)
    return got, st


def alone_by_recall(nets, r):
    """The same trajectory through axon_recall (plain method: one present launch)."""
    net = nets[r["net"]]
    cue = ax.clamp_words(r["cols"], net.ncol)[None, :]
    return net.recall(cue, CLAMP + r["free"], CLAMP, method="plain")["final"][0]


def test_mix_equals_alone(fleet):
    nets, pats = fleet
    reqs = requests(pats, 150, 1)
    mix, st = serve(nets, reqs)
    # about 50 trajectories per network per tick: the batched drive kernel runs; a request
    # served alone runs the gather kernel
    assert st["completed"] == 150 and st["max_batch"] > 3 * 24
    for r in reqs[:20]:
        alone, _ = serve(nets, [r])
        assert np.array_equal(alone[r["tag"]][1], mix[r["tag"]][1]), r["tag"]
    for r in reqs:
        assert np.array_equal(mix[r["tag"]][1], alone_by_recall(nets, r)), r["tag"]
        res = mix[r["tag"]][0]
        assert res["steps"] == CLAMP + r["free"] and res["net"] == r["net"]
        assert res["arrive_s"] <= res["admit_s"] <= res["done_s"]


def test_staggered_arrivals_and_few_slots(fleet):
    nets, pats = fleet
    reqs = requests(pats, 40, 2)
    base, _ = serve(nets, reqs)
    staggered, _ = serve(nets, reqs, spread_s=0.05)
    with ax.Server(nets, 16 << 20) as probe:
        cost = probe.stats()
    few, st = serve(nets, reqs, mem_bytes=cost["fixed_bytes"] + 3 * cost["slot_bytes"] + 100)
    assert st["slots"] == 3 and st["max_batch"] <= 3  # admission is bounded by the memory budget
    for r in reqs:
        t = r["tag"]
        assert np.array_equal(base[t][1], staggered[t][1]) and np.array_equal(base[t][1], few[t][1]), t


def test_bad_requests(fleet):
    nets, _ = fleet
    with ax.Server(nets, 16 << 20) as srv:
        with pytest.raises(ax._capi.AxonError):
            srv.submit(7, [1, 2], CLAMP, 5, 0)  # no such network
        with pytest.raises(ax._capi.AxonError):
            srv.submit(0, [64], CLAMP, 5, 0)  # not an input column
        with pytest.raises(ax._capi.AxonError):
            srv.submit(0, [1], 0, 0, 0)  # no steps
    with pytest.raises(ax._capi.AxonError):
        ax.Server(nets, 1024)  # budget below one slot


@pytest.mark.parametrize("variant", [dict(facil=40, ktest=5), dict(boost=2000), dict(mode=2, dthr=2, boost=0),
                                     dict(mode=0, dthr=3)])
def test_variants_in_the_mix_equal_recall(variant):
    """Readout variants through both drive kernels: facilitation (u32 counters in the
    batched kernel), drives past 16 bits (u32 slabs), the two-layer and point modes. Each
    request's final spikes equal axon_recall's for that network and cue."""
    cfg = dict(CFG, **variant)
    nets = [ax.Network(cfg) for _ in SEEDS]
    try:
        ax.multi_train(nets, SEEDS, LOADS, epochs=1, stimcols=STIMCOLS, readout=False, autotune=False, slots=3)
        pats = [ax.stimuli(s, L, 64, STIMCOLS) for s, L in zip(SEEDS, LOADS)]
        reqs = requests(pats, 110, 7)  # about 37 per network: the batched drive runs
        mix, st = serve(nets, reqs)
        assert st["max_batch"] > 3 * 24
        for r in reqs:
            assert np.array_equal(mix[r["tag"]][1], alone_by_recall(nets, r)), (variant, r["tag"])
    finally:
        for n in nets:
            n.close()


def test_long_requests_equal_long_batched_recall(fleet):
    """Requests longer than the 64 steps the per-step records hold (the server keeps none):
    their final spikes equal a batched axon_recall of the same length run alone and in a
    batch (the batched method takes up to 1024 steps when it keeps no per-step records),
    and the first 64 steps equal the plain method's."""
    nets, pats = fleet
    reqs = [dict(tag=i, net=i % 3, cols=np.sort(pats[i % 3][i % LOADS[i % 3]][: 4 + i]).astype(np.uint32), free=f)
            for i, f in enumerate([59, 60, 75, 123])]
    got, _ = serve(nets, reqs)
    for r in reqs:
        net = nets[r["net"]]
        cue = ax.clamp_words(r["cols"], net.ncol)[None, :]
        alone = net.recall(cue, CLAMP + r["free"], CLAMP)["final"][0]
        assert np.array_equal(got[r["tag"]][1], alone), r["tag"]
        batch = net.recall(np.repeat(cue, 5, axis=0), CLAMP + r["free"], CLAMP)["final"]
        assert all(np.array_equal(b, alone) for b in batch)
    r = reqs[0]  # 64 steps: also the plain method
    assert np.array_equal(got[r["tag"]][1], alone_by_recall(nets, r))
    from axon_b200._capi import AxonError

    with pytest.raises(AxonError):
        nets[0].recall(ax.clamp_words(reqs[2]["cols"], nets[0].ncol)[None, :], 80, CLAMP, hist=True)
