"""Failure detection of the persistent kernels without a GPU fault.

Every grid-wide wait is bounded. The host-side hook axon_inject_missing_arrival makes the
next launch wait at its barriers for a CTA that was never launched (as if one had died):
the wait runs out after the wait limit, every CTA returns, the host reads the error word
and reports AXON_ETIMEOUT, and the context stays usable - the same network presents
normally afterwards and matches one that never failed."""
import numpy as np
import pytest

import axon_b200 as ax
from axon_b200._capi import AXON_ETIMEOUT, AxonError

pytestmark = pytest.mark.gpu

CFG = dict(ax.CONFIG_C, ncol=512, incols=64, target=24)
SHORT_NS = 50_000_000  # 50 ms


def stim(seed=0):
    pats = ax.stimuli(seed, 3, 64, 16)
    return ax.load_stim(pats[0], 1.0, 1000, 512)


def test_present_barrier_timeout_is_reported_and_recoverable():
    with ax.Network(CFG) as net, ax.Network(CFG) as ref:
        net.init(0)
        ref.init(0)
        net.set_wait_limit(SHORT_NS)
        net.inject_missing_arrival(1)
        with pytest.raises(AxonError) as e:
            net.present(stim(), 10, 10, False)  # a readout: the aborted call changes no weight
        assert e.value.status == AXON_ETIMEOUT
        assert np.array_equal(net.read("W3"), ref.read("W3"))
        for n in (net, ref):  # the hook is one-shot: the next presentation runs normally
            n.present(stim(), 10, 5, True)
        assert np.array_equal(net.read("W3"), ref.read("W3"))
        assert np.array_equal(net.read("BIAS"), ref.read("BIAS"))
        a = net.recall(np.stack([stim()] * 4), 10, 5)["final"]
        b = ref.recall(np.stack([stim()] * 4), 10, 5)["final"]
        assert np.array_equal(a, b)


def test_multi_network_timeout_is_reported_and_recoverable():
    nets = [ax.Network(CFG) for _ in range(3)]
    try:
        nets[0].set_wait_limit(SHORT_NS)
        nets[0].inject_missing_arrival(1)
        with pytest.raises(AxonError) as e:
            ax.multi_train(nets, [0, 1, 2], [2, 3, 2], epochs=1, stimcols=16, autotune=False, slots=3)
        assert e.value.status == AXON_ETIMEOUT
        a, _ = ax.multi_train(nets, [0, 1, 2], [2, 3, 2], epochs=1, stimcols=16, autotune=False, slots=3)
        b, _ = ax.multi_train(nets, [0, 1, 2], [2, 3, 2], epochs=1, stimcols=16, method="plain")
        assert a == b
    finally:
        for n in nets:
            n.close()


def test_bad_hook_arguments():
    with ax.Network(CFG) as net:
        with pytest.raises(AxonError):
            net.inject_missing_arrival(0)
        with pytest.raises(AxonError):
            net.set_wait_limit(0)
