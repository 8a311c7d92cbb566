"""The `axon` command line against the oracle's: identical stdout, line for line, apart
from the banner's hardware name and wall-clock timings; and the published spot-check row
scraped exactly as the reference's bench/cap10.sh scrapes it."""
import json
import subprocess
from pathlib import Path

import pytest

import oracle_lib as O
from metrics import scrape

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
GOLD = json.loads((Path(__file__).parent / "golden" / "published.json").read_text())
CONFIG_C = GOLD["config_c"].split()
SMALL = ["ncol=512", "incols=64", "stimcols=16", "target=24"]


def engine_cli(args):
    from axon_b200 import build

    build.build_lib()
    exe = build.build_cli()
    p = subprocess.run([str(exe), *args], capture_output=True, text=True, timeout=1800)
    assert p.returncode == 0, p.stderr
    return p.stdout


def comparable(out: str) -> list[str]:
    keep = []
    for ln in out.splitlines():
        if ln.startswith(" AXON v0  -  columnar assembly engine"):
            continue
        if "ms/timestep" in ln or " st/s " in ln or "full step: serial" in ln:
            continue
        keep.append(ln)
    return keep


def assert_same(args):
    a, b = comparable(engine_cli(args)), comparable(O.run_cli(args))
    for i, (x, y) in enumerate(zip(a, b)):
        assert x == y, f"line {i}:\n engine: {x}\n oracle: {y}"
    assert len(a) == len(b)


@pytest.mark.parametrize("extra", [
    [*CONFIG_C, "stim=6", "epochs=3", "deep=1", "wave=1", "wavet=35", "split=1", "unionchar=1", "diag=1"],
    [*CONFIG_C, "stim=5", "epochs=2", "vbs=1", "vtopk=1", "ktest=8", "facil=3", "quiet=1"],
    ["stim=4", "epochs=2", "deep=1", "wave=1"],                      # the reference's built-in defaults
    [*CONFIG_C, "stim=3", "epochs=0", "deep=1", "margingate=1", "hetero=1", "seed=9"],
    [*CONFIG_C, "stim=7", "epochs=1", "T=20", "clampsteps=8", "trainclamp=6", "mode=0", "dthr=3", "wave=1",
     "wavet=60", "biasdownevery=3"],
    [*CONFIG_C, "stim=6", "epochs=3", "cueflip=25"],                  # the noisy-cue recall row (not a reference key)
    [*CONFIG_C, "stim=5", "epochs=2", "cueflip=10", "T=12"],
])
def test_cli_matches_oracle_small(extra):
    assert_same([*SMALL, *extra])


def test_cli_spot_check_full_size():
    args = [*CONFIG_C, "stim=12", "epochs=40", "deep=1", "wave=1", "wavet=35"]
    out = engine_cli(args)
    m = scrape(out)
    g = GOLD["spot_check"]
    assert (m["within_pct"], m["recall"], m["best_other"], m["sustained"], m["drive_t6"]) == (
        g["within_pct"], g["recall"], g["best_other"], g["sustained"], g["drive_t6"])
    ref = comparable(O.run_cli(args))
    assert comparable(out) == ref


def test_profile_mode_times_phases_and_changes_nothing_else():
    """profile=1 (the reference's per-kernel GPU profile, src/axon.mm:1161-1256) prints the
    per-phase device-timer profile of one learning presentation; it runs on a copy of the
    network, so every other line equals the run without it."""
    base = [*SMALL, *CONFIG_C, "stim=3", "epochs=1", "deep=1"]
    plain = comparable(engine_cli(base))
    out = engine_cli([*base, "profile=1"]).splitlines()
    i = next(k for k, ln in enumerate(out) if "PER-PHASE GPU PROFILE" in ln)
    j = next(k for k in range(i + 1, len(out)) if out[k].startswith("====="))
    rows = {ln[:42].strip(): ln[42:].split() for ln in out[i + 3:j - 3]}
    total = float(out[j - 3][42:].split()[0])
    parts = [float(v[0]) for v in rows.values()]
    assert len(parts) == 4 and all(p >= 0 for p in parts) and abs(sum(parts) - total) <= 0.05 * total + 0.5
    rest = out[:i - 1] + out[j + 1:]  # the profile block and the blank line before it
    assert comparable("\n".join(rest)) == plain
