"""The ctypes mirrors of the C ABI's structs have the header's layout: a small C program
built with gcc against include/axon_capi.h prints each struct's size and the offset of
every field, and the Python classes must agree field by field."""
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]

PAIRS = {  # ctypes class -> C type
    "AxonCfg": "axon_cfg",
    "RecallArgs": "axon_recall_args",
    "StateDev": "axon_state_dev",
    "MultiArgs": "axon_multi_args",
    "MultiResult": "axon_multi_result",
    "MultiReport": "axon_multi_report",
    "CkptMeta": "axon_ckpt_meta",
    "ServeResult": "axon_serve_result",
    "ServeCounters": "axon_serve_counters",
}


def test_ctypes_structs_match_header(tmp_path):
    import axon_b200._capi as A

    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "axon_capi.h"', "int main(void) {"]
    for py, c in PAIRS.items():
        cls = getattr(A, py)
        lines.append(f'  printf("{py} size %zu\\n", sizeof({c}));')
        for name, *_ in cls._fields_:
            lines.append(f'  printf("{py} {name} %zu\\n", offsetof({c}, {name}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    try:
        subprocess.run(["gcc", "-std=c11", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True,
                       capture_output=True, text=True)
    except FileNotFoundError:
        pytest.skip("gcc not available")
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for ln in out:
        if ln:
            py, field, val = ln.split()
            got[(py, field)] = int(val)
    for py in PAIRS:
        cls = getattr(A, py)
        assert got[(py, "size")] == __import__("ctypes").sizeof(cls), py
        for name, *_ in cls._fields_:
            assert got[(py, name)] == getattr(cls, name).offset, (py, name)
