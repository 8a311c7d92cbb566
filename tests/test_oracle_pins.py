"""Pins the CPU oracle to the reference's own known answers before anything is compared
with it: the bit-serial KAT (src/axon.mm:903-956), the serial/parallel top-K identity
(src/axon.mm:958-994), the k-WTA popcount KAT (bench/probe05_prop.mm:235-250) and the
published spot-check row and untrained control (README.md:58-66, tex:253-255)."""
import json
from pathlib import Path

import numpy as np
import pytest

import oracle_lib as O
from metrics import scrape

GOLD = json.loads((Path(__file__).parent / "golden" / "published.json").read_text())
CONFIG_C = GOLD["config_c"].split()


def planes_from_values(vals: np.ndarray) -> list[np.ndarray]:
    """4-bit values (one per synapse) -> 4 bitplanes of 32-bit words."""
    bits = [((vals >> b) & 1).astype(np.uint32) for b in range(4)]
    w = np.uint32(1) << np.arange(32, dtype=np.uint32)
    return [(b.reshape(-1, 32) * w).sum(axis=1, dtype=np.uint64).astype(np.uint32) for b in bits]


def values_from_planes(planes) -> np.ndarray:
    out = np.zeros(planes[0].size * 32, dtype=np.int64)
    for b, p in enumerate(planes):
        bits = (p[:, None] >> np.arange(32, dtype=np.uint32)) & 1
        out |= bits.reshape(-1).astype(np.int64) << b
    return out


@pytest.mark.parametrize("op,lo,hi", [(0, 0, 0), (1, 0, 0), (2, 5, 11), (2, 6, 10), (2, 4, 12)])
def test_bitserial_kat(oracle, op, lo, hi):
    # every (value, mask) pair, several times over, plus a random tail
    rng = np.random.default_rng(424242)
    vals = np.concatenate([np.tile(np.repeat(np.arange(16), 2), 64), rng.integers(0, 16, 1 << 16)])
    mask = np.concatenate([np.tile(np.tile([0, 1], 16), 64), rng.integers(0, 2, 1 << 16)])
    planes = planes_from_values(vals)
    mplane = planes_from_values(mask)[0]
    out = values_from_planes(O.bstest(op, lo, hi, planes, mplane))
    if op == 0:
        exp = np.where(mask == 1, np.minimum(15, vals + 1), vals)
    elif op == 1:
        exp = np.where(mask == 1, np.maximum(0, vals - 1), vals)
    else:
        exp = np.clip(vals, lo, hi)
    assert np.array_equal(out, exp)


def test_vbs_block_exact():
    out = O.run_cli(["vbs=1", "epochs=0", "stim=2", "ncol=256", "incols=64", "target=16", "stimcols=16", "quiet=1"])
    rows = [ln for ln in out.splitlines() if "values  mismatches" in ln]
    assert len(rows) == 5 and all(ln.rstrip().endswith("EXACT") for ln in rows)


def test_topk_serial_equals_parallel():
    out = O.run_cli(["vtopk=1", "epochs=0", "stim=4", "ncol=512", "incols=64", "target=16", "stimcols=16",
                     "quiet=1"])
    assert "BIT-IDENTICAL" in out and "mismatches 0" in out


@pytest.mark.parametrize("k", [1, 3, 5, 8, 16])
def test_kwta_popcount(oracle, k):
    # every ballot of a k-WTA column has exactly k bits (bench/probe05_prop.mm:235-250)
    import axon_b200._capi as A  # the cfg struct layout only; no GPU call

    c = A.AxonCfg()
    for f, v in dict(ncol=256, incols=64, inbr=4, nand=2, target=256, k=k, dthr=1, boost=4, mode=0, biasdown=1,
                     biasshift=4, biasdownevery=1, bandlo=5, bandhi=11, margingate=0, ltdrep=1, ltdevery=1,
                     topkpar=1).items():
        setattr(c, f, v)
    net = O.OracleNet(c, threads=4)
    net.init(3)
    stim = np.zeros(256, dtype=np.uint32)
    stim[np.arange(0, 64, 3)] = 0xFFFFFFFF
    net.present(stim, 2, 1, False)
    # target=256 exceeds the recurrent column count, so theta = 1 and every recurrent
    # column with drive >= 1 fires exactly its k winners at step 1 (written to SPK_A)
    spk = net.read("SPK_A")
    drive = net.read("DRIVE")
    pc = np.array([bin(int(x)).count("1") for x in spk[64:]])
    assert np.all(pc[drive[64:] >= 1] == k)


def test_untrained_control():
    out = O.run_cli([*CONFIG_C, "stim=12", "epochs=0", "deep=1"])
    m = scrape(out)
    assert m["within_pct"] == GOLD["untrained"]["within_pct"]
    assert m["drive_t6"] == GOLD["untrained"]["drive"]


def test_spot_check_row():
    """config C, 12 patterns, 40 epochs, seed 0: the row the reference's README requires."""
    out = O.run_cli([*CONFIG_C, "stim=12", "epochs=40", "deep=1", "wave=1", "wavet=35"])
    m = scrape(out)
    g = GOLD["spot_check"]
    assert (m["within_pct"], m["recall"], m["best_other"], m["sustained"], m["drive_t6"]) == (
        g["within_pct"], g["recall"], g["best_other"], g["sustained"], g["drive_t6"])


def test_table1_fixture_matches_paper():
    """The oracle's Table 1 run (tests/golden/oracle_table1.json, made by make_golden.py)
    reproduces every published seed-0 row, loads 12 to 300."""
    fx = json.loads((Path(__file__).parent / "golden" / "oracle_table1.json").read_text())
    assert sorted(int(k) for k in fx["rows"]) == sorted(r["stim"] for r in GOLD["table1"])
    for row in GOLD["table1"]:
        got = fx["rows"][str(row["stim"])]
        assert f"{float(got['within_pct']):.2f}" == row["within"]
        assert got["recall"] == row["recall"] and got["best_other"] == row["best_other"]
        assert got["margin"] == row["margin"] and got["sustained"] == row["sustained"]
        assert got["drive_t6"] == row["drive"]


@pytest.mark.slow
@pytest.mark.parametrize("stim", [24, 36, 48, 60])
def test_table1_row_regenerated(stim):
    out = O.run_cli([*CONFIG_C, f"stim={stim}", "epochs=40", "deep=1", "wave=1", "wavet=35"])
    m = scrape(out)
    row = next(r for r in GOLD["table1"] if r["stim"] == stim)
    assert f"{float(m['within_pct']):.2f}" == row["within"]
    assert (m["recall"], m["best_other"], m["margin"], m["sustained"], m["drive_t6"]) == (
        row["recall"], row["best_other"], row["margin"], row["sustained"], row["drive"])


def test_table2_fixture_matches_paper():
    """The oracle's five-seed runs (tests/golden/oracle_table2.json, made by make_golden.py),
    summarised as bench/seeds.sh summarises them, reproduce the published replication
    table (paper/axon_preprint.tex:288-292) and its 12-pattern sustained mean (:298-299)."""
    fx = json.loads((Path(__file__).parent / "golden" / "oracle_table2.json").read_text())
    t2 = GOLD["table2"]
    for row in t2["rows"]:
        got = fx["summary"][str(row["stim"])]
        for f in ("sustained_mean", "sustained_sd", "margin_mean", "margin_sd", "within_mean", "within_sd"):
            assert got[f] == row[f], (row["stim"], f, got[f], row[f])
    assert fx["summary"]["12"]["sustained_mean"] == t2["stim12_sustained_mean"]


def kwta_cases(seed=11):
    """Columns of 32 values for the k-of-32 known-answer tests: heavy ties (values 0..3),
    spread values, values at and above 2^27 and near 2^32, all-equal and all-zero columns,
    with every k from 0 to 33."""
    rng = np.random.default_rng(seed)
    cols, ks = [], []
    for k in range(34):
        for hi in (1, 4, 40, 1 << 16, 1 << 27, 1 << 32):
            for _ in range(6):
                cols.append(rng.integers(0, hi, 32, dtype=np.uint64).astype(np.uint32))
                ks.append(k)
        cols.append(np.full(32, 7, dtype=np.uint32)); ks.append(k)
        cols.append(np.zeros(32, dtype=np.uint32)); ks.append(k)
        big = rng.integers((1 << 27) - 3, (1 << 27) + 3, 32, dtype=np.uint64).astype(np.uint32)
        cols.append(big); ks.append(k)
    return np.stack(cols), np.array(ks, dtype=np.uint32)


def test_kwta_oracle_matches_rank_definition():
    """The oracle's k-of-32 (src/axon.mm:134-144) against the rank definition computed here:
    rank_i = #{j : v_j > v_i or (v_j == v_i and j < i)}, winners rank < k, vk and vk1 the
    values ranked k-1 and k."""
    v, ks = kwta_cases()
    got = O.kwtatest(v, ks)
    for i in range(len(ks)):
        x = v[i].astype(np.int64)
        rank = np.array([np.sum((x > x[a]) | ((x == x[a]) & (np.arange(32) < a))) for a in range(32)])
        k = int(ks[i])
        ball = sum(1 << a for a in range(32) if rank[a] < k)
        vk = int(x[rank == k - 1][0]) if k >= 1 and k <= 32 else 0
        vk1 = int(x[rank == k][0]) if k <= 31 else 0
        assert (int(got[i, 0]), int(got[i, 1]), int(got[i, 2])) == (ball, vk, vk1), (i, k)
