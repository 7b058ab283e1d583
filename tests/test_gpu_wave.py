"""The wavefront loop (kernel_mode 2: closest hit and physics as separate kernels over a pool of
paths in HBM) against the one-kernel persistent loop (kernel_mode 1): photons, seq, hits and
sensor counts bit for bit, with pool refill (more photons than pool slots), bounce and time caps,
event jumps and the batched multi-event form."""
import numpy as np
import pytest

from opticks_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def det(cuda):
    fd, lib, icdf = scenes.detector()
    phys = lib.arrays()
    phys["icdf"] = icdf
    return cuda, fd, lib, phys


def _engines(det, n, **kw):
    from opticks_b200 import engine as E
    torch, fd, lib, phys = det
    a = E.Engine(fd.arrays(), phys, E.default_config(max_photon=n, num_sensor=scenes.NUM_PMT, kernel_mode=1, **kw), device=0)
    b = E.Engine(fd.arrays(), phys, E.default_config(max_photon=n, num_sensor=scenes.NUM_PMT, kernel_mode=2, **kw), device=0)
    return a, b


def _run(torch, eng, g, N, ev):
    dev = g.device
    ph = torch.empty((N, 4, 4), dtype=torch.float32, device=dev)
    sq = torch.empty((N, 2, 2), dtype=torch.int64, device=dev)
    ht = torch.empty((N, 4, 4), dtype=torch.float32, device=dev)
    sn = torch.zeros((scenes.NUM_PMT,), dtype=torch.int32, device=dev)
    nh, st = eng.simulate_device(g, N, ev, photon=ph, seq=sq, hit=ht, hit_capacity=N, sensor_hits=sn,
                                 stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return ph, sq, ht[:nh], sn, st


@pytest.mark.parametrize("num_genstep,per,event,kw", [
    (20, 5000, 0, {}),
    (20, 5000, 3, {}),
    (300, 10000, 1, {"wave_pool": 1 << 20}),               # 3M photons through 1M slots: refill, then the tail
    (300, 10000, 1, {}),                                   # 3M photons, all in flight
    (40, 5000, 2, {"max_bounce": 3}),
    (40, 5000, 0, {"max_time": 40.0}),
])
def test_wave_equals_persistent(det, num_genstep, per, event, kw):
    torch = det[0]
    gs = scenes.detector_gensteps(num_genstep, per, seed=11, lib=det[2])
    N = num_genstep * per
    a, b = _engines(det, N, **kw)
    g = torch.from_numpy(gs).cuda()
    ra = _run(torch, a, g, N, event)
    rb = _run(torch, b, g, N, event)
    assert ra[4] == 0 and rb[4] == 0
    assert torch.equal(ra[0].view(torch.int32), rb[0].view(torch.int32))
    assert torch.equal(ra[1], rb[1])
    assert ra[2].shape[0] > 0
    assert torch.equal(ra[2].view(torch.int32), rb[2].view(torch.int32))
    assert torch.equal(ra[3], rb[3])
    a.close(); b.close()


@pytest.mark.parametrize("kw", [{}, {"wave_pool": 1 << 18}])      # all in flight; refill through 256k slots
def test_wave_batched_equals_persistent(det, kw):
    torch = det[0]
    gs = scenes.batched_events(64, median=20000.0, lib=det[2])
    ev = np.arange(len(gs), dtype=np.int32)
    counts = gs.view(np.int32)[:, 0, 3].astype(np.int64)
    N = int(counts.sum())
    a, b = _engines(det, int(counts.max()), **kw)
    g = torch.from_numpy(gs).cuda()
    e = torch.from_numpy(ev).cuda()
    outs = []
    for eng in (a, b):
        ph = torch.empty((N, 4, 4), dtype=torch.float32, device="cuda")
        sq = torch.empty((N, 2, 2), dtype=torch.int64, device="cuda")
        nh, st = eng.simulate_batched_device(g, e, N, photon=ph, seq=sq, stream=torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        assert st == 0
        outs.append((ph, sq))
    assert torch.equal(outs[0][0].view(torch.int32), outs[1][0].view(torch.int32))
    assert torch.equal(outs[0][1], outs[1][1])
    a.close(); b.close()


@pytest.mark.parametrize("launch", [dict(wave_rounds=3, use_graph=1, wave_refill=8),
                                    dict(wave_rounds=10, use_graph=1, wave_refill=32),
                                    dict(wave_rounds=0, wave_tail=1 << 12, wave_refill=1)])
def test_wave_schedules_equal_persistent(det, launch):
    """the autotuner's knobs change no result: a fixed schedule of rounds then the tail kernel,
    captured as a CUDA graph and replayed (second call), other refill thresholds, another tail
    threshold; batched and plain calls"""
    torch = det[0]
    gs = scenes.batched_events(48, median=20000.0, lib=det[2])
    ev = np.arange(len(gs), dtype=np.int32)
    counts = gs.view(np.int32)[:, 0, 3].astype(np.int64)
    N = int(counts.sum())
    a, b = _engines(det, int(counts.max()))
    b.set_launch_config(**launch)
    g = torch.from_numpy(gs).cuda()
    e = torch.from_numpy(ev).cuda()
    outs = []
    for eng, calls in ((a, 1), (b, 2)):
        ph = torch.empty((N, 4, 4), dtype=torch.float32, device="cuda")
        sq = torch.empty((N, 2, 2), dtype=torch.int64, device="cuda")
        for _ in range(calls):
            ph.fill_(0.0)
            nh, st = eng.simulate_batched_device(g, e, N, photon=ph, seq=sq, stream=torch.cuda.current_stream().cuda_stream)
            torch.cuda.synchronize()
            assert st == 0
        outs.append((ph, sq))
    assert torch.equal(outs[0][0].view(torch.int32), outs[1][0].view(torch.int32))
    assert torch.equal(outs[0][1], outs[1][1])
    # plain call of one event with the same launch shape (a fixed schedule applies to batched calls only)
    g1 = torch.from_numpy(np.ascontiguousarray(gs[:3])).cuda()
    n1 = int(counts[:3].sum())
    ra, rb = _run(torch, a, g1, n1, 7), _run(torch, b, g1, n1, 7)
    assert rb[4] == 0
    assert torch.equal(ra[0].view(torch.int32), rb[0].view(torch.int32))
    assert torch.equal(ra[1], rb[1]) and torch.equal(ra[3], rb[3])
    a.close(); b.close()


def test_wave_batched_beyond_minimum_pool_equals_persistent(det):
    """84M photons in one batched call with wave_pool left at 0: more than the 2^26-slot minimum
    pool, so the slot count comes from the free device memory (every photon in flight here);
    photons, seq and hit count bit for bit against the persistent loop"""
    torch = det[0]
    gs = scenes.batched_events(1024, median=50000.0, lib=det[2])
    ev = np.arange(len(gs), dtype=np.int32)
    counts = gs.view(np.int32)[:, 0, 3].astype(np.int64)
    N = int(counts.sum())
    assert N > (1 << 26)
    a, b = _engines(det, int(counts.max()))
    g = torch.from_numpy(gs).cuda()
    e = torch.from_numpy(ev).cuda()
    outs = []
    for eng in (a, b):
        ph = torch.empty((N, 4, 4), dtype=torch.float32, device="cuda")
        sq = torch.empty((N, 2, 2), dtype=torch.int64, device="cuda")
        nh, st = eng.simulate_batched_device(g, e, N, photon=ph, seq=sq, stream=torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        assert st == 0
        outs.append((ph, sq, nh))
        eng.close()
    assert torch.equal(outs[0][0].view(torch.int32), outs[1][0].view(torch.int32))
    assert torch.equal(outs[0][1], outs[1][1])
    assert outs[0][2] == outs[1][2]
    del outs
    torch.cuda.empty_cache()
