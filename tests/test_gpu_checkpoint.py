"""Network checkpoints (axon_save / axon_load): a trained network written to a file and read
into a fresh network gives back the same state and the same readouts; a corrupt, truncated
or mismatched file is refused before the network changes."""
import numpy as np
import pytest

import axon_b200 as ax
from axon_b200._capi import AxonError

pytestmark = pytest.mark.gpu

CFG = dict(ax.CONFIG_C, ncol=512, incols=64, target=24)
STATE = ("W0", "W1", "W2", "W3", "CONN", "BIAS", "MULT")


def trained(seed=3, nstim=4):
    net = ax.Network(CFG)
    net.init(seed)
    pats = ax.stimuli(seed, nstim, 64, 16)
    for ep in range(2):
        for p in range(nstim):
            net.present(ax.load_stim(pats[p], 1.0, 1000 + p, 512), 10, 5, True)
    return net, pats


def test_round_trip(tmp_path):
    net, pats = trained()
    path = tmp_path / "net.axck"
    net.save(path, seed=3, nstim=4, stimcols=16, epochs=2)
    with ax.Network(CFG) as other:
        meta = other.load(path)
        assert meta == {"seed": 3, "nstim": 4, "stimcols": 16, "epochs": 2}
        for b in STATE:
            assert np.array_equal(net.read(b), other.read(b)), b
        cues = np.stack([ax.load_stim(pats[q], 0.75, 4400 + q, 512) for q in range(4)])
        a = net.recall(cues, 10, 5)["final"]
        b = other.recall(cues, 10, 5)["final"]
        assert np.array_equal(a, b)
        for n in (net, other):  # training continues identically from the loaded state
            n.present(ax.load_stim(pats[0], 1.0, 1000, 512), 10, 5, True)
        for b in STATE:
            assert np.array_equal(net.read(b), other.read(b)), b
    net.close()


def test_refuses_bad_files(tmp_path):
    net, _ = trained()
    path = tmp_path / "net.axck"
    net.save(path, seed=3, nstim=4, stimcols=16, epochs=2)
    raw = path.read_bytes()
    with ax.Network(CFG) as other:
        other.init(9)
        before = other.read("W3")
        bad = bytearray(raw)
        bad[len(raw) // 2] ^= 0x01
        (tmp_path / "flip.axck").write_bytes(bytes(bad))
        (tmp_path / "short.axck").write_bytes(raw[: len(raw) - 100])
        for name in ("flip.axck", "short.axck", "missing.axck"):
            with pytest.raises(AxonError):
                other.load(tmp_path / name)
        assert np.array_equal(other.read("W3"), before)  # a refused load changes nothing
    with ax.Network(dict(CFG, k=12)) as different:
        with pytest.raises(AxonError):
            different.load(path)
    net.close()
