"""Genstep slices with photon offsets on the GPU reproduce the whole event bit for bit (the
multi-GPU split, run here as successive slices on one GPU), and the event-sharded adjoint equals
the mean of the per-event passes."""
import numpy as np
import pytest

from opticks_b200 import shard

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def det(cuda):
    import torch
    from opticks_b200 import engine as E
    from opticks_b200 import scenes
    fd, lib, icdf = scenes.detector()
    phys = lib.arrays()
    phys["icdf"] = icdf
    gs = scenes.detector_gensteps(12, 2000, seed=4, lib=lib)
    gs.view(np.int32)[:, 0, 3] = [2000, 150, 3100, 0, 900, 2500, 1800, 40, 2222, 1300, 700, 2600]
    eng = E.Engine(fd.arrays(), phys, E.default_config(max_photon=100_000, num_sensor=scenes.NUM_PMT), device=0)
    yield torch, eng, gs, lib, phys
    eng.close()


@pytest.mark.parametrize("parts", [2, 3, 5])
def test_slices_equal_whole_event(det, parts):
    torch, eng, gs, _, _ = det
    dev = torch.device("cuda", 0)
    fn = shard.engine_slice_fn(eng, dev, num_sensor=eng.num_sensor)
    N = int(shard.genstep_counts(gs).sum())
    whole = fn(gs, 3, 0, N)
    outs = [fn(gs[g0:g1], 3, off, n) for g0, g1, off, n in shard.genstep_slices(shard.genstep_counts(gs), parts)]
    torch.cuda.synchronize()
    photon = torch.cat([o["photon"] for o in outs])
    seq = torch.cat([o["seq"] for o in outs])
    hit = torch.cat([o["hit"] for o in outs])
    sens = sum(o["sensor_hits"] for o in outs)
    assert torch.equal(photon.view(torch.int32), whole["photon"].view(torch.int32))
    assert torch.equal(seq, whole["seq"])
    assert whole["hit"].shape[0] > 0
    assert torch.equal(hit.view(torch.int32), whole["hit"].view(torch.int32))
    assert torch.equal(sens, whole["sensor_hits"])


def test_event_sharded_adjoint_is_mean(det):
    torch, eng, gs, lib, phys = det
    from opticks_b200 import adjoint as ADJ
    dev = torch.device("cuda", 0)
    ml = lib.material_line("LS")
    th = ADJ.nominal_theta(phys, ml)
    H, J = shard.adjoint_sharded(eng, gs, [2, 5, 9], th, ml, 300.0, 620.0, dev)
    N = int(shard.genstep_counts(gs).sum())
    g = torch.from_numpy(gs).to(dev)
    h1 = torch.zeros_like(H)
    j1 = torch.zeros_like(J)
    hs, js = torch.zeros_like(H), torch.zeros_like(J)
    for ev in (2, 5, 9):
        ADJ.adjoint_device(eng, g, N, ev, th, ml, 300.0, 620.0, h1, j1, torch.cuda.current_stream(dev).cuda_stream)
        hs += h1
        js += j1
    torch.cuda.synchronize()
    assert H.sum().item() > 0
    assert torch.allclose(H, hs / 3, rtol=0, atol=0)
    assert torch.allclose(J, js / 3, rtol=1e-12, atol=1e-12)
