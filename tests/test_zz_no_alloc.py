"""axon_present_static: the allocation-free presentation entry point.

Hosts that own all device memory themselves (a framework's caching allocator, a service
that forbids allocation after start-up) cannot let the library cudaMalloc during a call.
This test hands the entry point buffers allocated by the caller (here by torch), runs two
presentations in a row through it and through the ordinary axon_present on an axon_net
holding the same state, and requires every output buffer to agree bit for bit - the same
exact-integer bar as every other parity test. Collected last so a failure here leaves the
rest of the suite already run.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NAMES = {  # axon_state_dev field -> axon_buf name
    "w0": "W0", "w1": "W1", "w2": "W2", "w3": "W3", "conn": "CONN", "bias": "BIAS", "mult": "MULT",
    "refball": "REFBALL", "stim": "STIM", "spk_a": "SPK_A", "spk_b": "SPK_B", "drive": "DRIVE", "bbits": "BBITS",
    "acc": "ACC", "marg": "MARG", "drive_log": "DRIVELOG", "stats": "STATS", "hist": "HIST", "theta": "THETA",
}
COMPARE = ["W0", "W1", "W2", "W3", "BIAS", "SPK_A", "SPK_B", "DRIVE", "BBITS", "ACC", "MARG", "DRIVELOG", "STATS"]


def device_copy(net):
    import torch

    bufs = {}
    for field, name in NAMES.items():
        host = net.read(name)
        bufs[field] = torch.from_numpy(host.view(np.int32)).cuda()
    return bufs


def static_present(cfg, bufs, stim, T, clamp, learn, use_bias) -> int:
    """One call through the C ABI; returns the change in free device memory across it."""
    import torch

    from axon_b200 import _capi as A

    bufs["stim"].copy_(torch.from_numpy(np.ascontiguousarray(stim, dtype=np.uint32).view(np.int32)))
    st = A.StateDev(**{f: C.c_void_p(bufs[f].data_ptr()) for f in NAMES})
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    A.check(A.lib().axon_present_static(C.byref(cfg), C.byref(st), T, clamp, int(learn), use_bias))
    free1 = torch.cuda.mem_get_info()[0]
    torch.cuda.synchronize()
    return free1 - free0


@pytest.mark.parametrize("geometry", ["small", "full"])
def test_static_present_matches_present(geometry):
    import axon_b200 as ax

    kw = dict(ax.CONFIG_C)
    if geometry == "small":
        kw.update(ncol=256, incols=64, target=16, k=12)
    cfg = ax.config(**kw)
    net = ax.Network(cfg)
    net.init(1)
    pats = ax.stimuli(1, 4, cfg.incols, 16 if geometry == "small" else 64)
    for p in range(2):
        net.present(ax.load_stim(pats[p], 1.0, 1000 + p, cfg.ncol), 10, 5, True)
    ref = net.final_spikes(10)
    net.write("REFBALL", ref)
    bufs = device_copy(net)
    calls = [(ax.load_stim(pats[2], 1.0, 1002, cfg.ncol), 10, 5, True, 2),
             (ax.load_stim(pats[3], 0.75, 4403, cfg.ncol), 35, 5, False, 0)]
    for i, (stim, T, clamp, learn, ub) in enumerate(calls):
        net.present(stim, T, clamp, learn, True, ub)
        delta = static_present(cfg, bufs, stim, T, clamp, learn, ub)
        if i > 0:  # the first call on the device may load the module; later calls allocate nothing
            assert delta == 0, f"call {i}: free device memory changed by {delta} bytes"
        for name in COMPARE + ["HIST", "THETA"]:
            field = next(f for f, n in NAMES.items() if n == name)
            got = bufs[field].cpu().numpy().view(np.uint32)
            exp = net.read(name)
            if name == "HIST":
                got, exp = got[: T * cfg.ncol], exp[: T * cfg.ncol]
            if name == "THETA":
                got, exp = got[:1], exp[:1]
            assert np.array_equal(got, exp), f"call {i}: {name} differs in {np.count_nonzero(got != exp)} words"


def test_static_present_rejects_oversized_network():
    import axon_b200 as ax
    from axon_b200 import _capi as A

    cfg = ax.config(**dict(ax.CONFIG_C, ncol=8192))
    st = A.StateDev(**{f: C.c_void_p(16) for f in NAMES})  # never dereferenced: rejected first
    status = A.lib().axon_present_static(C.byref(cfg), C.byref(st), 10, 5, 0, 0)
    assert status == A.AXON_EINVAL
    assert b"4096" in A.lib().axon_last_error()


def test_static_present_rejects_misaligned_pointer():
    """The planes are read as 16-byte vectors and W3 tiles are bulk-copied, so a pointer
    that is not 16-byte aligned is refused before anything is launched."""
    import torch

    import axon_b200 as ax
    from axon_b200 import _capi as A

    cfg = ax.config(**dict(ax.CONFIG_C, ncol=256, incols=64, target=16, k=12))
    buf = torch.zeros(64, dtype=torch.int32, device="cuda")
    ptrs = {f: C.c_void_p(buf.data_ptr()) for f in NAMES}
    ptrs["w3"] = C.c_void_p(buf.data_ptr() + 4)  # never dereferenced: rejected first
    st = A.StateDev(**ptrs)
    status = A.lib().axon_present_static(C.byref(cfg), C.byref(st), 10, 5, 0, 0)
    assert status == A.AXON_EINVAL
    assert b"16-byte aligned" in A.lib().axon_last_error()
