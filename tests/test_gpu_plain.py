"""GPU parity of the plain path: every buffer of the CUDA engine equals the CPU oracle's,
word for word, after init and after every presentation (integer state: bit-exact)."""
import numpy as np
import pytest

import oracle_lib as O

pytestmark = pytest.mark.gpu

BUFS_EACH_PRESENT = ["SPK_A", "SPK_B", "DRIVE", "BBITS", "ACC", "BIAS", "MARG", "DRIVELOG", "STATS", "STIM"]


def make_cfg(**kw):
    import axon_b200 as ax

    base = dict(ncol=256, incols=64, inbr=4, nand=4, target=16, k=12, dthr=1, mode=1, contrast=1, margingate=0,
                ltdrep=1, ltdevery=2, biasup=73, biasdown=1)
    base.update(kw)
    return ax.config(**base)


def compare(gpu, cpu, names, T=None, where=""):
    for nm in names:
        g, c = gpu.read(nm), cpu.read(nm)
        if nm == "HIST" and T is not None:
            g, c = g[: T * gpu.ncol], c[: T * gpu.ncol]
        if not np.array_equal(g, c):
            bad = np.flatnonzero(g != c)
            raise AssertionError(f"{where}: {nm} differs at {bad.size} words, first {bad[:5]}: "
                                 f"gpu {g[bad[:5]]} cpu {c[bad[:5]]}")
    th_g, th_c = gpu.read("THETA")[0], cpu.read("THETA")[0]
    assert th_g == th_c, f"{where}: theta {th_g} vs {th_c}"


def planes_equal(gpu, cpu, where=""):
    for p in ("W0", "W1", "W2", "W3"):
        g, c = gpu.read(p), cpu.read(p)
        assert np.array_equal(g, c), f"{where}: plane {p} differs at {np.count_nonzero(g != c)} words"


def run_protocol(cfgkw, nstim=4, epochs=2, T=10, clamp=5, stimcols=16, seed=0, check_planes_every=1):
    import axon_b200 as ax

    cfg = make_cfg(**cfgkw)
    gpu = ax.Network(cfg)
    cpu = O.OracleNet(cfg)
    gpu.init(seed)
    cpu.init(seed)
    planes_equal(gpu, cpu, "init")
    compare(gpu, cpu, ["CONN"], where="init")
    pats = ax.stimuli(seed, nstim, cfg.incols, stimcols)
    n = 0
    for ep in range(epochs):
        for p in range(nstim):
            stim = ax.load_stim(pats[p], 1.0, 1000 + p, cfg.ncol)
            gpu.present(stim, T, clamp, True)
            cpu.present(stim, T, clamp, True)
            where = f"learn ep{ep} p{p}"
            compare(gpu, cpu, BUFS_EACH_PRESENT + ["HIST"], T=T, where=where)
            n += 1
            if n % check_planes_every == 0:
                planes_equal(gpu, cpu, where)
    planes_equal(gpu, cpu, "after training")
    # readouts: cue fractions, bias on/off, longer free runs with a logged reference assembly
    ref = gpu.final_spikes(T)
    gpu.write("REFBALL", ref)
    cpu.write("REFBALL", ref)
    mult = np.random.default_rng(1).integers(0, 3, cfg.ncol * 32).astype(np.uint32)
    gpu.write("MULT", mult)
    cpu.write("MULT", mult)
    for q, keep, ub, TT in [(0, 1.0, 2, T), (1, 0.75, 0, T), (2, 0.5, 1, T), (3 % nstim, 0.25, 0, 35), (0, 0.0, 0, 30)]:
        stim = ax.load_stim(pats[q], keep, 4400 + q, cfg.ncol)
        gpu.present(stim, TT, clamp, False, True, ub)
        cpu.present(stim, TT, clamp, False, True, ub)
        compare(gpu, cpu, BUFS_EACH_PRESENT + ["HIST"], T=TT, where=f"readout q{q} keep{keep} bias{ub}")
    return gpu, cpu


def test_bitserial_kat_gpu():
    import axon_b200 as ax

    rng = np.random.default_rng(7)
    n = 1 << 14
    for op, lo, hi in [(0, 0, 0), (1, 0, 0), (2, 5, 11), (2, 6, 10), (2, 4, 12)]:
        planes = [rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32) for _ in range(4)]
        mask = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
        exp = O.bstest(op, lo, hi, [p.copy() for p in planes], mask)
        got = [p.copy() for p in planes]
        ax.bstest(op, lo, hi, got, mask)
        for e, g in zip(exp, got):
            assert np.array_equal(e, g)


def test_init_matches_oracle_full_geometry():
    import axon_b200 as ax

    cfg = ax.config(**ax.CONFIG_C)
    gpu = ax.Network(cfg)
    cpu = O.OracleNet(cfg)
    for seed in (0, 5):
        gpu.init(seed)
        cpu.init(seed)
        planes_equal(gpu, cpu, f"init seed {seed}")
        compare(gpu, cpu, ["CONN"], where="init")
        assert gpu.wstat() == cpu.wstat()


def test_config_c_small_geometry():
    run_protocol({})


@pytest.mark.parametrize("variant", [
    dict(margingate=1),
    dict(contrast=0),                       # legacy rule: inc + depress on odd steps
    dict(hetero=1, ltdrep=2, ltdevery=1),
    dict(mode=0, dthr=2),
    dict(mode=2, dthr=3, boost=7),
    dict(topkpar=0, target=24),
    dict(biasdownevery=3, biasshift=2, ktest=8, facil=5),
    dict(target=0),
    dict(target=250),                       # more than the recurrent columns: theta = 1
    dict(k=32, target=40),
    dict(k=0),
])
def test_variants_small_geometry(variant):
    run_protocol(variant, nstim=3, epochs=1)


def test_config_c_full_geometry_one_epoch():
    """Full 131,072-neuron network, config C: one training epoch of 12 patterns and
    readouts, all state compared after every presentation."""
    import axon_b200 as ax

    run_protocol(dict(ncol=4096, incols=512, target=64, k=24), nstim=12, epochs=1, stimcols=64, check_planes_every=4)


def test_diagnostics_match_oracle():
    import axon_b200 as ax

    gpu, cpu = run_protocol({}, nstim=3, epochs=1)
    ncol = gpu.ncol
    ball = gpu.final_spikes(10)
    mult = gpu.read("MULT")
    for um in (0, 1):
        post = (np.arange(ncol * 32) % 3 == 0).astype(np.uint32)
        assert np.array_equal(gpu.within(ball, um, post, mult), cpu.within(ball, um, post, mult))
    assert np.array_equal(gpu.within(ball), cpu.within(ball))
    assert np.array_equal(gpu.indeg(), cpu.indeg())
    assert np.array_equal(gpu.untouched(), cpu.untouched())
    assert gpu.wstat() == cpu.wstat()
    memb = np.random.default_rng(2).integers(0, 8, ncol * 32).astype(np.uint32)
    asm = np.stack([ball, np.roll(ball, 8), np.roll(ball, 16)]).astype(np.uint32)
    for sel in (0, 1, 2):
        assert np.array_equal(gpu.wdiag(memb, asm, 3, sel), cpu.wdiag(memb, asm, 3, sel))


@pytest.mark.parametrize("ncol", [8192, 4608])
def test_widest_network_two_columns_per_warp(ncol):
    """ncol 8,192, the widest network the engine takes, runs k_present with 2 columns per
    warp (the grid must fit one wave of co-resident CTAs), and so does 4,608, where one
    column per warp would need more than 28 warps per CTA: learning and readout
    presentations against the oracle; a wider network is refused at creation."""
    import axon_b200 as ax

    with pytest.raises(ax._capi.AxonError):
        ax.Network(make_cfg(ncol=16384, incols=512))

    cfg = make_cfg(ncol=ncol, incols=512, target=64, k=24)
    gpu = ax.Network(cfg)
    cpu = O.OracleNet(cfg)
    gpu.init(5)
    cpu.init(5)
    pats = ax.stimuli(5, 2, cfg.incols, 64)
    for p in range(2):
        stim = ax.load_stim(pats[p], 1.0, 1000 + p, cfg.ncol)
        gpu.present(stim, 8, 4, True)
        cpu.present(stim, 8, 4, True)
        compare(gpu, cpu, BUFS_EACH_PRESENT + ["HIST"], T=8, where=f"ncol {ncol} learn p{p}")
    planes_equal(gpu, cpu, f"ncol {ncol}")
    stim = ax.load_stim(pats[1], 0.75, 4401, cfg.ncol)
    gpu.present(stim, 12, 4, False, True, 0)
    cpu.present(stim, 12, 4, False, True, 0)
    compare(gpu, cpu, BUFS_EACH_PRESENT + ["HIST"], T=12, where=f"ncol {ncol} readout")
    gpu.close()
    cpu.close()


@pytest.mark.parametrize("T,clamp", [(1, 0), (1, 1), (64, 0), (64, 64), (3, 2)])
def test_step_count_limits(T, clamp):
    """The shortest and longest presentations (T = 1 and T = 64, the hist capacity), with
    no clamped step and with every step clamped."""
    import axon_b200 as ax

    cfg = make_cfg()
    gpu = ax.Network(cfg)
    cpu = O.OracleNet(cfg)
    gpu.init(2)
    cpu.init(2)
    pats = ax.stimuli(2, 2, cfg.incols, 16)
    for learn in (True, False):
        stim = ax.load_stim(pats[0], 1.0, 1000, cfg.ncol)
        gpu.present(stim, T, clamp, learn)
        cpu.present(stim, T, clamp, learn)
        compare(gpu, cpu, BUFS_EACH_PRESENT + ["HIST"], T=T, where=f"T{T} clamp{clamp} learn{learn}")
    planes_equal(gpu, cpu, f"T{T}")
    gpu.close()
    cpu.close()


@pytest.mark.parametrize("target,inbr", [(1500, 4), (64, 32)])
def test_dense_activity_overflows_tile_pool(target, inbr):
    """Nearly every branch non-silent: a CTA's columns need far more W3 tiles than its
    shared-memory tile pool holds, so most columns stream their tiles through registers,
    and the threshold bin holds many drives. Learning and readout against the oracle."""
    import axon_b200 as ax

    cfg = make_cfg(ncol=4096, incols=512, inbr=inbr, target=target, k=24)
    gpu = ax.Network(cfg)
    cpu = O.OracleNet(cfg)
    gpu.init(7)
    cpu.init(7)
    pats = ax.stimuli(7, 2, cfg.incols, 448)
    for p in range(2):
        stim = ax.load_stim(pats[p], 1.0, 1000 + p, cfg.ncol)
        gpu.present(stim, 6, 3, True)
        cpu.present(stim, 6, 3, True)
        compare(gpu, cpu, BUFS_EACH_PRESENT + ["HIST"], T=6, where=f"dense learn p{p}")
    planes_equal(gpu, cpu, "dense")
    stim = ax.load_stim(pats[0], 0.5, 4400, cfg.ncol)
    gpu.present(stim, 8, 3, False, True, 0)
    cpu.present(stim, 8, 3, False, True, 0)
    compare(gpu, cpu, BUFS_EACH_PRESENT + ["HIST"], T=8, where="dense readout")
    gpu.close()
    cpu.close()


def test_kwta_kat_gpu():
    """The kernels' k-of-32 (bit-sliced rank) equals the oracle's on ties, spread values and
    values up to 2^32 - 1, for every k from 0 to 33."""
    import axon_b200 as ax
    from test_oracle_pins import kwta_cases

    v, ks = kwta_cases()
    assert np.array_equal(ax.kwtatest(v, ks), O.kwtatest(v, ks))
