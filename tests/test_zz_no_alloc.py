"""The allocation-free entry point phx_simulate_device_noalloc, called through the C ABI.

Some callers of this library cannot allocate device memory on each call: a framework whose
caching allocator owns all device memory, or a per-event loop that cannot take the device-wide
synchronisation cudaMalloc/cudaFree may imply.  This entry point keeps its scratch in one fixed
device array inside the library.  Its results must equal those of phx_simulate_device on the
same inputs, on two calls in a row (the array keeps the previous call's contents, so anything
it fails to clear would show up in the second call)."""
import ctypes as C

import numpy as np
import pytest

from opticks_b200 import scenes

pytestmark = pytest.mark.gpu


def _ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _run(fn, eng, g, G, N, event, bufs, torch):
    from opticks_b200._lib import PhxOutputs
    for t in bufs.values():
        t.fill_(7)          # stale contents must be overwritten
    out = PhxOutputs(_ptr(bufs["photon"]), _ptr(bufs["seq"]), _ptr(bufs["hit"]), N, _ptr(bufs["sensor"]), 0, 0, 0)
    rc = fn(eng._h, _ptr(g), G, N, event, 0, C.byref(out), None)
    if rc != 0:
        from opticks_b200 import _lib
        raise RuntimeError(_lib.lib().phx_last_error().decode())
    torch.cuda.synchronize()
    nh = int(out.num_hit)
    return dict(photon=bufs["photon"].cpu().numpy(), seq=bufs["seq"].cpu().numpy(),
                hit=bufs["hit"][:nh].cpu().numpy(), sensor=bufs["sensor"].cpu().numpy(),
                num_hit=nh, status=int(out.status))


@pytest.fixture(scope="module")
def setup(cuda):
    torch = cuda
    from opticks_b200 import engine as E
    fd, lib, icdf = scenes.detector()
    phys = lib.arrays()
    phys["icdf"] = icdf
    gs = scenes.detector_gensteps(3, 2000, seed=4, lib=lib)
    N = int(gs.view(np.int32)[:, 0, 3].sum())
    eng = E.Engine(fd.arrays(), phys, E.default_config(max_photon=N, num_sensor=scenes.NUM_PMT))
    dev = torch.device("cuda", 0)
    g = torch.from_numpy(gs).to(dev)

    def bufs():
        return dict(photon=torch.empty((N, 4, 4), dtype=torch.float32, device=dev),
                    seq=torch.empty((N, 2, 2), dtype=torch.int64, device=dev),
                    hit=torch.empty((N, 4, 4), dtype=torch.float32, device=dev),
                    sensor=torch.empty((scenes.NUM_PMT,), dtype=torch.int32, device=dev))
    yield torch, eng, g, len(gs), N, bufs
    eng.close()


def test_noalloc_matches_the_allocating_entry_point_twice(setup):
    from opticks_b200 import _lib
    torch, eng, g, G, N, bufs = setup
    L = _lib.lib()
    ref = _run(L.phx_simulate_device, eng, g, G, N, 3, bufs(), torch)
    assert ref["status"] == 0 and ref["num_hit"] > 0
    b = bufs()
    for call in range(2):
        got = _run(L.phx_simulate_device_noalloc, eng, g, G, N, 3, b, torch)
        assert got["status"] == ref["status"], call
        assert got["num_hit"] == ref["num_hit"], call
        # same kernels on the same inputs: equal within the parity tolerance, in fact bit for bit
        np.testing.assert_array_equal(got["photon"], ref["photon"])
        np.testing.assert_array_equal(got["seq"], ref["seq"])
        np.testing.assert_array_equal(got["hit"], ref["hit"])
        np.testing.assert_array_equal(got["sensor"], ref["sensor"])


def test_noalloc_rejects_sizes_beyond_its_limit(setup):
    from opticks_b200 import _lib
    from opticks_b200._lib import PhxOutputs
    torch, eng, g, G, N, bufs = setup
    L = _lib.lib()
    out = PhxOutputs(None, None, None, 0, None, 0, 0, 0)
    rc = L.phx_simulate_device_noalloc(eng._h, _ptr(g), G, (1 << 23) + 1, 0, 0, C.byref(out), None)
    assert rc != 0 and b"limit" in L.phx_last_error()
    rc = L.phx_simulate_device_noalloc(eng._h, _ptr(g), G, N, 0, 1 << 22, C.byref(out), None)
    assert rc != 0 and b"RNG slots" in L.phx_last_error()
