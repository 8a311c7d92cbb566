"""GPU parity of the batched readout: each of B trajectories of axon_recall equals the
oracle's present(learn=0) for that cue (final spikes, every step's spikes, k_emit
counters, member-drive log), for the batched and the plain method."""
import numpy as np
import pytest

import oracle_lib as O

pytestmark = pytest.mark.gpu


def trained_pair(cfgkw, nstim, epochs, stimcols, seed=0):
    import axon_b200 as ax

    base = dict(ncol=256, incols=64, inbr=4, nand=4, target=16, k=12, dthr=1, mode=1, contrast=1, margingate=0,
                ltdrep=1, ltdevery=2, biasup=73, biasdown=1)
    base.update(cfgkw)
    cfg = ax.config(**base)
    gpu = ax.Network(cfg)
    gpu.init(seed)
    pats = ax.stimuli(seed, nstim, cfg.incols, stimcols)
    for _ in range(epochs):
        for p in range(nstim):
            gpu.present(ax.load_stim(pats[p], 1.0, 1000 + p, cfg.ncol), 10, 5, True)
    cpu = O.OracleNet(cfg)
    for name in ("W0", "W1", "W2", "W3", "CONN", "BIAS"):
        cpu.write(name, gpu.read(name))
    return cfg, gpu, cpu, pats


def make_cues(pats, ncol, B, rng):
    import axon_b200 as ax

    keeps = [1.0, 0.75, 0.5, 0.35, 0.25, 0.1, 0.0]
    return np.stack([ax.load_stim(pats[b % len(pats)], keeps[b % len(keeps)], 4400 + b, ncol) for b in range(B)])


def oracle_runs(cpu, cues, T, clamp, use_bias, ref=None):
    finals, hists, stats, logs = [], [], [], []
    for b in range(cues.shape[0]):
        cpu.write("DRIVELOG", np.zeros(256, dtype=np.uint32))
        cpu.write("REFBALL", ref[b] if ref is not None else np.zeros(cues.shape[1], dtype=np.uint32))
        cpu.present(cues[b], T, clamp, False, True, use_bias)
        finals.append(cpu.read("SPK_B" if T & 1 else "SPK_A"))
        hists.append(cpu.read("HIST")[: T * cues.shape[1]].reshape(T, -1))
        stats.append(cpu.read("STATS"))
        logs.append(cpu.read("DRIVELOG"))
    return np.stack(finals), np.stack(hists), np.stack(stats), np.stack(logs)


@pytest.mark.parametrize("method", ["batched", "plain"])
@pytest.mark.parametrize("B,T,clamp,use_bias", [(1, 10, 5, 0), (7, 10, 5, 1), (40, 35, 5, 0), (33, 45, 10, 0)])
def test_recall_matches_oracle_small(method, B, T, clamp, use_bias):
    cfg, gpu, cpu, pats = trained_pair({}, 6, 3, 16)
    rng = np.random.default_rng(B)
    cues = make_cues(pats, cfg.ncol, B, rng)
    ref = np.stack([gpu.final_spikes(10)] * B)
    mult = rng.integers(0, 3, cfg.ncol * 32).astype(np.uint32)
    gpu.write("MULT", mult)
    cpu.write("MULT", mult)
    r = gpu.recall(cues, T, clamp, use_bias=use_bias, method=method, hist=True, stats=True, ref_ball=ref)
    f, h, s, dl = oracle_runs(cpu, cues, T, clamp, use_bias, ref)
    assert np.array_equal(r["final"], f)
    assert np.array_equal(r["hist"], h)
    if method == "batched":  # word 2 (branch coincidence) is produced by the plain method only
        s = s.copy()
        s[:, 2] = 0
        r["stats"][:, 2] = 0
    assert np.array_equal(r["stats"], s)
    assert np.array_equal(r["drive_log"], dl)


@pytest.mark.parametrize("variant", [dict(mode=0, dthr=2), dict(mode=2, dthr=0, boost=9), dict(ktest=5, facil=40),
                                     dict(topkpar=0, target=0), dict(target=300), dict(boost=2000), dict(incols=20)])
def test_recall_variants(variant):
    cfg, gpu, cpu, pats = trained_pair(variant, 4, 2, 16)
    cues = make_cues(pats, cfg.ncol, 9, np.random.default_rng(0))
    r = gpu.recall(cues, 20, 5, hist=True)
    f, h, _, _ = oracle_runs(cpu, cues, 20, 5, 0)
    assert np.array_equal(r["final"], f)
    assert np.array_equal(r["hist"], h)


def test_recall_batched_equals_plain_full_geometry():
    """Config C network at full size (131,072 neurons): batched and plain readouts of
    60 cues agree word for word, and a sample of trajectories matches the oracle."""
    import axon_b200 as ax

    cfg, gpu, cpu, pats = trained_pair(dict(ncol=4096, incols=512, target=64, k=24), 12, 2, 64)
    cues = make_cues(pats, cfg.ncol, 60, np.random.default_rng(1))
    rb = gpu.recall(cues, 45, 10, hist=True)
    rp = gpu.recall(cues, 45, 10, hist=True, method="plain")
    assert np.array_equal(rb["final"], rp["final"])
    assert np.array_equal(rb["hist"], rp["hist"])
    idx = [0, 13, 59]
    f, h, _, _ = oracle_runs(cpu, cues[idx], 45, 10, 0)
    assert np.array_equal(rb["final"][idx], f)
    assert np.array_equal(rb["hist"][idx], h)


@pytest.mark.parametrize("B", [149, 320, 400])
def test_recall_several_trajectories_per_cta(B):
    """More trajectories than CTAs (one per SM, 148 on a B200): a CTA's warp groups each
    select the threshold of a trajectory of their own, some groups taking a second whole
    trajectory or a part of one, the next one's drives loading while the current one is
    processed. At 400 trajectories two counter buffers no longer fit in shared memory, and
    phase 1 keeps one with a second barrier per item. Every trajectory equals the plain
    method; a sample, including later trajectories, equals the oracle."""
    cfg, gpu, cpu, pats = trained_pair({}, 6, 3, 16)
    cues = make_cues(pats, cfg.ncol, B, np.random.default_rng(B))
    rb = gpu.recall(cues, 20, 5, hist=True, stats=True)
    rp = gpu.recall(cues, 20, 5, hist=True, method="plain")
    assert np.array_equal(rb["final"], rp["final"])
    assert np.array_equal(rb["hist"], rp["hist"])
    idx = [0, 148, B - 1]
    f, h, s, _ = oracle_runs(cpu, cues[idx], 20, 5, 0)
    assert np.array_equal(rb["final"][idx], f)
    assert np.array_equal(rb["hist"][idx], h)
    s = s.copy()
    s[:, 2] = 0  # branch coincidence: plain method only
    st = rb["stats"][idx].copy()
    st[:, 2] = 0
    assert np.array_equal(st, s)


def test_batched_equals_plain_at_the_widest_batched_network():
    """ncol = 8,192, the widest network the batched kernel takes (the plain path at that
    width is checked against the oracle in test_gpu_plain): both methods agree on every
    trajectory's spikes at every step. 160 trajectories put two on some CTAs; at this
    width the threshold step has room for one drive buffer only."""
    import axon_b200 as ax

    cfg = ax.config(ncol=8192, incols=512, **ax.CONFIG_C)
    with ax.Network(cfg) as net:
        net.init(4)
        pats = ax.stimuli(4, 6, 512, 64)
        for p in range(6):
            net.present(ax.load_stim(pats[p], 1.0, 1000 + p, 8192), 10, 5, True)
        cues = np.stack([ax.load_stim(pats[q % 6], 0.6 + 0.05 * (q % 5), 4400 + q, 8192) for q in range(160)])
        a = net.recall(cues, 25, 6, hist=True)
        b = net.recall(cues, 25, 6, hist=True, method="plain")
        assert np.array_equal(a["hist"], b["hist"]) and np.array_equal(a["final"], b["final"])


def test_graph_replay_equals_direct_launch():
    """graph=1 captures the batched launch once and replays it while the arguments repeat;
    the results equal a direct launch, also after the weights change (the tile layout is
    rebuilt in place, so the replayed graph reads the new weights)."""
    import axon_b200 as ax

    cfg, gpu, cpu, pats = trained_pair({}, 4, 1, 16)
    cues = make_cues(pats, cfg.ncol, 12, np.random.default_rng(3))
    direct = gpu.recall(cues, 20, 5, hist=True)
    g1 = gpu.recall(cues, 20, 5, hist=True, graph=True)  # captured
    g2 = gpu.recall(cues, 20, 5, hist=True, graph=True)  # replayed
    for r in (g1, g2):
        assert np.array_equal(r["hist"], direct["hist"]) and np.array_equal(r["final"], direct["final"])
    gpu.present(ax.load_stim(pats[0], 1.0, 1000, cfg.ncol), 10, 5, True)
    after = gpu.recall(cues, 20, 5, hist=True)
    g3 = gpu.recall(cues, 20, 5, hist=True, graph=True)
    assert np.array_equal(g3["hist"], after["hist"])


def test_final_spikes_into_caller_array():
    """final_out: the final spikes land in the caller's array (page-locked here, as a
    serving host would pass it), equal to a recall that allocates its own result."""
    import torch

    cfg, gpu, cpu, pats = trained_pair({}, 3, 1, 16)
    cues = make_cues(pats, cfg.ncol, 9, np.random.default_rng(4))
    want = gpu.recall(cues, 12, 5)["final"]
    buf = torch.zeros(cues.shape, dtype=torch.int32).pin_memory().numpy().view(np.uint32)
    for graph in (False, True, True):
        r = gpu.recall(cues, 12, 5, graph=graph, final_out=buf)
        assert r["final"] is buf and np.array_equal(buf, want)
        buf[:] = 0
    with pytest.raises(AssertionError):
        gpu.recall(cues, 12, 5, final_out=np.zeros((cues.shape[0], cfg.ncol), dtype=np.int32))


@pytest.mark.parametrize("variant", [{}, dict(mode=0, dthr=2), dict(mode=2, dthr=0, boost=9), dict(ktest=5, facil=40),
                                     dict(boost=2000)])
def test_tensor_contraction_matches_oracle(variant):
    """contraction="tensor" (binary MMA on the tensor cores) gives every trajectory the same
    spikes at every step as the CUDA-core popcounts and as the oracle, packed 16-bit counters
    and 32-bit ones (boost=2000) alike, with multi-word entries (clamped input groups)."""
    cfg, gpu, cpu, pats = trained_pair(variant, 6, 2, 16)
    cues = make_cues(pats, cfg.ncol, 37, np.random.default_rng(5))
    rt = gpu.recall(cues, 20, 5, hist=True, stats=True, contraction="tensor")
    rp = gpu.recall(cues, 20, 5, hist=True, stats=True)
    assert np.array_equal(rt["hist"], rp["hist"]) and np.array_equal(rt["stats"], rp["stats"])
    f, h, _, _ = oracle_runs(cpu, cues[:5], 20, 5, 0)
    assert np.array_equal(rt["hist"][:5], h) and np.array_equal(rt["final"][:5], f)


def test_tensor_contraction_full_geometry():
    """Config C at full size, 300 cues of 45 steps: the tensor contraction equals the
    CUDA-core one on every trajectory and step (several trajectories per CTA included)."""
    cfg, gpu, cpu, pats = trained_pair(dict(ncol=4096, incols=512, target=64, k=24), 12, 2, 64)
    cues = make_cues(pats, cfg.ncol, 300, np.random.default_rng(2))
    rt = gpu.recall(cues, 45, 10, hist=True, contraction="tensor")
    rp = gpu.recall(cues, 45, 10, hist=True)
    assert np.array_equal(rt["hist"], rp["hist"])


@pytest.mark.parametrize("variant", [{}, dict(mode=0, dthr=2), dict(mode=2, dthr=0, boost=9), dict(incols=24)])
def test_slab_policies_match_oracle(variant):
    """Which per-neuron drives the batched kernel stores does not change any result: storing
    only those at or above each trajectory's histogram floor ("floor", the default, and
    "floor_always", where every drive drop below the floor goes through the recompute)
    gives the same spikes and counters at every step as storing all ("full"), and the
    oracle's."""
    cfg, gpu, cpu, pats = trained_pair(variant, 6, 2, 16)
    cues = make_cues(pats, cfg.ncol, 37, np.random.default_rng(6))
    runs = {s: gpu.recall(cues, 20, 5, hist=True, stats=True, slab=s) for s in ("full", "floor", "floor_always")}
    for s in ("floor", "floor_always"):
        assert np.array_equal(runs[s]["hist"], runs["full"]["hist"]), s
        assert np.array_equal(runs[s]["stats"], runs["full"]["stats"]), s
    f, h, _, _ = oracle_runs(cpu, cues[:5], 20, 5, 0)
    assert np.array_equal(runs["floor_always"]["hist"][:5], h)


@pytest.mark.parametrize("contraction", ["popc", "tensor"])
def test_slab_policies_full_geometry(contraction):
    """Config C at full size, 300 cues of 45 steps: the three slab policies agree on every
    trajectory and step (at the step after the clamp almost every trajectory's threshold
    falls below its floor, so "floor_always" recomputes many gated columns there)."""
    cfg, gpu, cpu, pats = trained_pair(dict(ncol=4096, incols=512, target=64, k=24), 12, 2, 64)
    cues = make_cues(pats, cfg.ncol, 300, np.random.default_rng(3))
    runs = {s: gpu.recall(cues, 45, 10, hist=True, stats=True, contraction=contraction, slab=s)
            for s in ("full", "floor", "floor_always")}
    for s in ("floor", "floor_always"):
        assert np.array_equal(runs[s]["hist"], runs["full"]["hist"]), s
        assert np.array_equal(runs[s]["stats"], runs["full"]["stats"]), s


@pytest.mark.parametrize("B,T,clamp", [(1, 1, 1), (5, 1, 0), (9, 7, 0), (9, 6, 6), (37, 12, 2), (530, 6, 3)])
def test_recall_edge_shapes(B, T, clamp):
    """One-step readouts, no clamped step, every step clamped, the afferent cache's shortest
    clamp (2 steps), and more trajectories than one launch holds (512: the host splits the
    batch): the batched method equals the plain one on every trajectory and step, and a
    sample equals the oracle."""
    cfg, gpu, cpu, pats = trained_pair({}, 6, 3, 16)
    cues = make_cues(pats, cfg.ncol, B, np.random.default_rng(B + T))
    rb = gpu.recall(cues, T, clamp, hist=True, stats=True)
    rp = gpu.recall(cues, T, clamp, hist=True, stats=True, method="plain")
    assert np.array_equal(rb["hist"], rp["hist"]) and np.array_equal(rb["final"], rp["final"])
    idx = sorted({0, B // 2, B - 1})
    f, h, _, _ = oracle_runs(cpu, cues[idx], T, clamp, 0)
    assert np.array_equal(rb["hist"][idx], h) and np.array_equal(rb["final"][idx], f)


def test_recall_refuses_bad_arguments():
    """The recall refuses, with AXON_EINVAL and before any copy or launch, an unknown slab
    policy or contraction unit, T = 0, T above 64 with per-step records or above 1024
    without, and B = 0; the network stays usable."""
    import ctypes as C

    import axon_b200._capi as A

    cfg, gpu, cpu, pats = trained_pair({}, 2, 1, 16)
    cues = make_cues(pats, cfg.ncol, 3, np.random.default_rng(9))
    final = np.zeros_like(cues)
    for fields in (dict(slab=3), dict(contraction=2), dict(T=0)):
        a = A.RecallArgs(T=fields.get("T", 10), clamp_steps=5, slab=fields.get("slab", 0),
                         contraction=fields.get("contraction", 0))
        st = A.lib().axon_recall(gpu._h, cues.ctypes.data_as(C.c_void_p), 3, C.byref(a), None,
                                 final.ctypes.data_as(C.c_void_p), None, None, None, None)
        assert st == A.AXON_EINVAL, fields
    for T, hist in ((65, True), (1025, False)):
        with pytest.raises(A.AxonError) as e:
            gpu.recall(cues, T, 5, hist=hist)
        assert e.value.status == A.AXON_EINVAL
    with pytest.raises(A.AxonError) as e:
        gpu.recall(cues[:0], 10, 5)
    assert e.value.status == A.AXON_EINVAL
    f, _, _, _ = oracle_runs(cpu, cues[:1], 10, 5, 0)
    assert np.array_equal(gpu.recall(cues, 10, 5)["final"][:1], f)
