"""Batched persistent form: many uneven events in one launch (work queue + lane refill), captured as a
CUDA graph.  Each event's photons must equal that event simulated alone with phx_simulate_device
(same RNG slots and skipahead), to the parity bar; replays of the graph are deterministic."""
import numpy as np
import pytest

from opticks_b200 import scenes
from tests._parity import frac_close, seq_match

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def batch(cuda):
    torch = cuda
    from opticks_b200 import engine as E
    fd, lib, icdf = scenes.detector()
    phys = lib.arrays()
    phys["icdf"] = icdf
    counts = [1500, 37, 0, 4000, 900, 2500, 1, 3000, 700, 64]
    gs_list, ev = [], []
    rng = np.random.default_rng(3)
    matline = lib.material_line("LS")
    for e, n in enumerate(counts):
        # events 3 and 7 have two gensteps each
        parts = [n // 2, n - n // 2] if e in (3, 7) else [n]
        for m in parts:
            pos = scenes.uniform_ball(1, 17000.0, rng)[0]
            gs_list.append(scenes.scint_genstep(m, pos, matline))
            ev.append(e)
    gs = np.stack(gs_list)
    ev = np.array(ev, np.int32)
    N = int(sum(counts))
    eng = E.Engine(fd.arrays(), phys, E.default_config(max_photon=max(counts), num_sensor=scenes.NUM_PMT))
    dev = torch.device("cuda", 0)
    g = torch.from_numpy(gs).to(dev)
    gev = torch.from_numpy(ev).to(dev)
    photon = torch.zeros((N, 4, 4), dtype=torch.float32, device=dev)
    seq = torch.zeros((N, 2, 2), dtype=torch.int64, device=dev)
    hit = torch.zeros((N, 4, 4), dtype=torch.float32, device=dev)
    done = torch.zeros((len(counts) + 1,), dtype=torch.int64, device=dev)
    nh, st = eng.simulate_batched_device(g, gev, N, photon=photon, seq=seq, hit=hit, hit_capacity=N,
                                         num_event=len(counts), event_done_ns=done)
    res = dict(photon=photon.cpu().numpy(), seq=seq.cpu().numpy().view(np.uint64), hit=hit[:nh].cpu().numpy(),
               num_hit=nh, status=st, done=done.cpu().numpy())
    yield dict(torch=torch, eng=eng, gs=gs, ev=ev, counts=counts, N=N, res=res, g=g, gev=gev, dev=dev)
    eng.close()


def test_batched_equals_per_event_launches(batch):
    from opticks_b200 import engine as E
    r = batch["res"]
    assert r["status"] == 0, E.status_names(r["status"])
    off = np.concatenate([[0], np.cumsum(batch["counts"])])
    eng, gs, ev = batch["eng"], batch["gs"], batch["ev"]
    allp, alls = [], []
    for e, n in enumerate(batch["counts"]):
        sel = gs[ev == e]
        out = eng.simulate(sel, e)
        allp.append(out["photon"])
        alls.append(out["seq"])
    P, S = np.concatenate(allp), np.concatenate(alls)
    m = seq_match(r["seq"], S)
    same = np.all(r["seq"][:, 0, :] == S[:, 0, :], axis=1)
    fc = frac_close(r["photon"], P, same, 1e-4)
    exact = float(np.mean(np.all(r["photon"].view(np.uint32) == P.view(np.uint32), axis=(1, 2))))
    print(f"batched vs per-event: seqhis {m:.6f} close {fc:.6f} bit-exact {exact:.6f}")
    assert m >= 0.999 and fc >= 0.999
    # sphoton.index restarts at 0 in every event
    idx = r["photon"].view(np.uint32)[:, 3, 2]
    for e in range(len(batch["counts"])):
        np.testing.assert_array_equal(idx[off[e]:off[e + 1]], np.arange(batch["counts"][e], dtype=np.uint32))
    # hits are the SD photons of the concatenation in order
    flags = r["photon"].view(np.uint32)[:, 3, 3]
    np.testing.assert_array_equal(r["hit"], r["photon"][(flags & 0x40) != 0])


def test_batched_event_completion_times(batch):
    d = batch["res"]["done"]
    start = d[-1]
    for e, n in enumerate(batch["counts"]):
        if n > 0:
            assert d[e] >= start > 0
        else:
            assert d[e] == 0


def test_batched_graph_replay_is_deterministic(batch):
    torch = batch["torch"]
    N = batch["N"]
    photon = torch.zeros((N, 4, 4), dtype=torch.float32, device=batch["dev"])
    seq = torch.zeros((N, 2, 2), dtype=torch.int64, device=batch["dev"])
    outs = []
    for rep in range(3):
        photon.fill_(3.0)
        nh, st = batch["eng"].simulate_batched_device(batch["g"], batch["gev"], N, photon=photon, seq=seq)
        outs.append(photon.cpu().numpy().copy())
    np.testing.assert_array_equal(outs[0], outs[1])
    np.testing.assert_array_equal(outs[0], outs[2])
    np.testing.assert_array_equal(outs[0], batch["res"]["photon"])


def test_persistent_plain_mode_matches_one_thread_per_photon(cuda):
    from opticks_b200 import engine as E
    fd, lib, icdf = scenes.detector()
    phys = lib.arrays()
    phys["icdf"] = icdf
    gs = scenes.detector_gensteps(3, 1500, seed=9, lib=lib)
    a = E.Engine(fd.arrays(), phys, E.default_config(max_photon=4500, kernel_mode=0))
    b = E.Engine(fd.arrays(), phys, E.default_config(max_photon=4500, kernel_mode=1, block=64, regroup=2, chunk=1))
    ra, rb = a.simulate(gs, 2), b.simulate(gs, 2)
    a.close(); b.close()
    assert seq_match(ra["seq"], rb["seq"]) >= 0.999
    same = np.all(ra["seq"][:, 0, :] == rb["seq"][:, 0, :], axis=1)
    assert frac_close(ra["photon"], rb["photon"], same, 1e-4) >= 0.999
    assert abs(ra["num_hit"] - rb["num_hit"]) <= 3
