"""Regenerates tests/golden/oracle_table1.json: the CPU oracle's five measurements for
config C at loads 12..60 (seed 0, 40 epochs, deep=1 wave=1 wavet=35), as the reference's
bench/cap10.sh scrapes them. Run from the repository root:

    python tests/golden/make_golden.py            # runs the oracle CLI (~15 min on 8 cores)
    python tests/golden/make_golden.py --reuse D  # scrape saved stdout D/spot<load>.txt instead
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))

import oracle_lib as O  # noqa: E402
from metrics import scrape  # noqa: E402

LOADS = [12, 24, 36, 48, 60]


def main() -> None:
    gold = json.loads((HERE / "published.json").read_text())
    cfg = gold["config_c"].split()
    reuse = Path(sys.argv[sys.argv.index("--reuse") + 1]) if "--reuse" in sys.argv else None
    rows = {}
    for n in LOADS:
        args = [*cfg, f"stim={n}", "epochs=40", "deep=1", "wave=1", "wavet=35"]
        out = (reuse / f"spot{n}.txt").read_text() if reuse else O.run_cli(args)
        m = scrape(out)
        m.pop("steps_per_s", None)
        rows[str(n)] = m
    fx = {"generator": "tests/golden/make_golden.py", "oracle": "oracle/_build/axon_oracle",
          "args": cfg + ["stim=<load>", "epochs=40", "deep=1", "wave=1", "wavet=35"], "rows": rows}
    (HERE / "oracle_table1.json").write_text(json.dumps(fx, indent=1) + "\n")
    print(json.dumps(rows, indent=1))


if __name__ == "__main__":
    main()
