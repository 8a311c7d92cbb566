"""CPU checks of the C-ABI library: it loads without a GPU, exports every function the
public header declares, and its host-side stimulus stream matches the oracle's."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import oracle_lib as O

ROOT = Path(__file__).resolve().parents[1]


def header_functions() -> list[str]:
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        src = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"\b(axon_[a-z0-9_]+)\s*\(", src))
    return sorted(names)


@pytest.fixture(scope="module")
def capi():
    from axon_b200 import build

    build.build_lib()
    from axon_b200 import _capi

    return _capi.lib()


def test_library_exports_header(capi):
    names = header_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(capi, n)]
    assert not missing, missing


@pytest.mark.parametrize("seed,nstim,incols,stimcols", [(0, 12, 512, 64), (3, 60, 512, 64), (7, 5, 100, 37),
                                                         (1, 4, 64, 64), (2, 3, 9, 1)])
def test_stimulus_patterns_match_oracle(capi, seed, nstim, incols, stimcols):
    import axon_b200 as ax

    assert np.array_equal(ax.stimuli(seed, nstim, incols, stimcols), O.stimuli(seed, nstim, incols, stimcols))


@pytest.mark.parametrize("keep", [1.0, 0.75, 0.5, 0.35, 0.25, 0.15, 0.10, 0.05, 0.02, 0.0])
def test_load_stim_matches_oracle(capi, keep):
    import axon_b200 as ax

    pats = O.stimuli(0, 12, 512, 64)
    for q in range(12):
        for sd in (4400 + q, 5000 + q * 16 + 3, 999):
            assert np.array_equal(ax.load_stim(pats[q], keep, sd, 4096), O.load_stim(pats[q], keep, sd, 4096))


def test_bad_config_is_an_error_not_an_exit(capi):
    import axon_b200 as ax
    from axon_b200._capi import AxonError

    with pytest.raises(AxonError):
        ax.Network(ax.config(ncol=100))  # not a multiple of 32
    with pytest.raises(AxonError):
        ax.Network(ax.config(ncol=256, incols=256))


@pytest.mark.parametrize("frac", [0.0, 0.10, 0.25, 0.5, 1.0])
def test_noisy_cue_matches_oracle(capi, frac):
    """axon_noisy_cue against the oracle's own restatement, and its defining properties:
    only active bits are flipped, exactly round(frac * 32 * ncols) of them, and a smaller
    fraction flips a subset of a larger one's bits for the same seed."""
    import axon_b200 as ax

    pats = O.stimuli(0, 60, 512, 64)
    for q in (0, 17, 59):
        for pct, d in ((10, 0), (10, 1), (25, 0), (25, 1)):
            sd = ax.noisy_cue_seed(q, pct, d)
            assert sd == O.noisy_seed(q, pct, d) == 90000 + 1000 * pct + 16 * q + d
            got = ax.noisy_cue(pats[q], frac, sd, 4096)
            assert np.array_equal(got, O.noisy_cue(pats[q], frac, sd, 4096))
            full = ax.clamp_words(pats[q], 4096)
            assert np.all(got & ~full == 0)  # only active bits change
            flipped = int(np.bitwise_count(full).sum() - np.bitwise_count(got).sum())
            assert flipped == int(np.floor(frac * 64 * 32 + 0.5))
            if frac < 1.0:
                more = ax.noisy_cue(pats[q], min(1.0, frac + 0.25), sd, 4096)
                assert np.all(more & ~got == 0)  # the larger fraction's flips include these


def test_noisy_cue_rejects_bad_input(capi):
    import axon_b200 as ax
    from axon_b200._capi import AxonError

    with pytest.raises(AxonError):
        ax.noisy_cue(np.array([3, 3], dtype=np.uint32), 0.1, 1, 64)  # repeated column
    with pytest.raises(AxonError):
        ax.noisy_cue(np.array([70], dtype=np.uint32), 0.1, 1, 64)  # column out of range
    with pytest.raises(AxonError):
        ax.noisy_cue(np.array([1], dtype=np.uint32), 1.5, 1, 64)  # fraction above 1


def test_oracle_config_defaults_match_engine_defaults(capi):
    """The oracle's restated CLI defaults and the engine's axon_cfg_defaults agree field for
    field, with and without overrides (the reference arm builds its configuration from the
    oracle's alone)."""
    import axon_b200 as ax

    for kw in ({}, dict(ncol=4096, incols=512, **ax.CONFIG_C)):
        o, e = O.config(**kw), ax.config(**kw)
        for f in O.CFG_FIELDS:
            assert getattr(o, f) == getattr(e, f), f
