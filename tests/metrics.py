"""Extraction of the five published measurements from the CLI's stdout, with the same
patterns as the reference's bench/cap10.sh:15-24 (grep/awk restated in Python)."""
from __future__ import annotations

import re


def scrape(out: str) -> dict:
    lines = out.splitlines()
    m = {}
    for ln in lines:
        if "within-assembly :" in ln:
            g = re.search(r"= ([0-9.]+)%", ln)
            m["within_pct"] = g.group(1)
    for i, ln in enumerate(lines):
        if "pattern completion with bias OFF" in ln:
            for ln2 in lines[i + 1:i + 5]:
                if ln2.startswith("   75%"):
                    f = ln2.split()
                    m["recall"], m["best_other"], m["margin"] = f[2], f[3], f[4]
            break
    for i, ln in enumerate(lines):
        if "free-phase drive" in ln and i + 1 < len(lines):
            for tok in lines[i + 1].split():
                if tok.startswith("t6:"):
                    m["drive_t6"] = tok.split(":")[1]
            break
    free = []
    inwave = False
    for ln in lines:
        if "WAVE:" in ln:
            inwave = True
            continue
        if inwave:
            if ln.startswith("====="):
                break
            f = ln.split()
            if len(f) > 4 and f[1] == "FREE":
                free.append(f[4])
    if free:
        m["sustained"] = f"{float(free[-1]) / float(free[0]):.3f}"
    for ln in lines:
        g = re.search(r"->\s*([0-9]+) steps/s", ln)
        if g:
            m["steps_per_s"] = g.group(1)
            break
    return m


def seeds_summary(per_seed: list[dict]) -> dict:
    """Five-seed summary as the reference's bench/seeds.sh computes it: each seed's
    sustained ratio (printed with %.3f), margin and within-assembly density as printed;
    mean and sample standard deviation of each, printed with the script's formats."""
    import statistics as st

    v = [float(m["sustained"]) for m in per_seed]
    mg = [float(m["margin"]) for m in per_seed]
    d = [float(m["within_pct"]) for m in per_seed]
    return {"sustained_mean": f"{st.mean(v):.3f}", "sustained_sd": f"{st.stdev(v):.3f}",
            "margin_mean": f"{st.mean(mg):+.3f}", "margin_sd": f"{st.stdev(mg):.3f}",
            "within_mean": f"{st.mean(d):.2f}", "within_sd": f"{st.stdev(d):.2f}",
            "sustained_cv_pct": f"{100 * st.stdev(v) / st.mean(v):.1f}"}
