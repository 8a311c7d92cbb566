"""Regenerates the oracle's golden fixtures from its command line, as the reference's
bench scripts scrape the reference's:

* tests/golden/oracle_table1.json: the five measurements for config C, seed 0, 40 epochs,
  deep=1 wave=1 wavet=35 at every load of the published capacity sweep (12..300;
  bench/cap10.sh).
* tests/golden/oracle_table2.json: the same measurements for seeds 0-4 at loads
  12, 24, 36, 42, 48, 60 (bench/seeds.sh), with the per-load means and sample standard
  deviations computed as bench/seeds.sh computes them.

Run from the repository root:

    python tests/golden/make_golden.py                 # runs the oracle CLI (hours on 8 cores)
    python tests/golden/make_golden.py --save D        # also keeps each run's stdout in D/
    python tests/golden/make_golden.py --reuse D       # scrape saved stdout D/s<seed>_<load>.txt
    python tests/golden/make_golden.py --only table1   # one of the two fixtures

With --save, runs whose stdout is already in D are not repeated.
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))

import oracle_lib as O  # noqa: E402
from metrics import scrape, seeds_summary  # noqa: E402

TABLE1_LOADS = [12, 24, 36, 48, 60, 74, 90, 140, 200, 300]
TABLE2_LOADS = [12, 24, 36, 42, 48, 60]
TABLE2_SEEDS = [0, 1, 2, 3, 4]


def run(cfg: list[str], seed: int, load: int, save: Path | None, reuse: Path | None) -> dict:
    name = f"s{seed}_{load}.txt"
    src = reuse or save
    if src is not None and (src / name).exists():
        out = (src / name).read_text()
    else:
        if reuse is not None:
            raise FileNotFoundError(reuse / name)
        out = O.run_cli([*cfg, f"stim={load}", "epochs=40", f"seed={seed}", "deep=1", "wave=1", "wavet=35"])
        if save is not None:
            save.mkdir(parents=True, exist_ok=True)
            (save / name).write_text(out)
    m = scrape(out)
    m.pop("steps_per_s", None)
    return m


def main() -> None:
    gold = json.loads((HERE / "published.json").read_text())
    cfg = gold["config_c"].split()
    arg = lambda k: Path(sys.argv[sys.argv.index(k) + 1]) if k in sys.argv else None  # noqa: E731
    reuse, save = arg("--reuse"), arg("--save")
    only = sys.argv[sys.argv.index("--only") + 1] if "--only" in sys.argv else None
    common = {"generator": "tests/golden/make_golden.py", "oracle": "oracle/_build/axon_oracle",
              "args": cfg + ["stim=<load>", "epochs=40", "seed=<seed>", "deep=1", "wave=1", "wavet=35"]}
    if only in (None, "table1"):
        rows = {str(n): run(cfg, 0, n, save, reuse) for n in TABLE1_LOADS}
        (HERE / "oracle_table1.json").write_text(json.dumps({**common, "rows": rows}, indent=1) + "\n")
        print(json.dumps(rows, indent=1))
    if only in (None, "table2"):
        runs = {str(n): {str(s): run(cfg, s, n, save, reuse) for s in TABLE2_SEEDS} for n in TABLE2_LOADS}
        summ = {n: seeds_summary(list(r.values())) for n, r in runs.items()}
        (HERE / "oracle_table2.json").write_text(json.dumps({**common, "runs": runs, "summary": summ}, indent=1) + "\n")
        print(json.dumps(summ, indent=1))


if __name__ == "__main__":
    main()
