"""Sharding of the photon path across ranks (CPU: gloo, world_size 2).

The per-rank compute in the gloo tests is the CPU oracle (the checker), so these tests pin the
host logic of opticks_b200.shard: genstep slicing with photon offsets, the rank-order hit gather
and the per-sensor sum reproduce the single-process event exactly.
"""
import os
import socket

import numpy as np
import pytest

from opticks_b200 import shard

SD = 0x40


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_genstep_slices_cover_and_balance():
    rng = np.random.default_rng(3)
    for G in (1, 2, 7, 100):
        counts = rng.integers(0, 5000, size=G)
        total = int(counts.sum())
        for parts in (1, 2, 3, 4, 8):
            sl = shard.genstep_slices(counts, parts)
            assert len(sl) == parts
            assert sl[0][0] == 0 and sl[-1][1] == G
            off = 0
            for p, (g0, g1, o, n) in enumerate(sl):
                if p:
                    assert g0 == sl[p - 1][1]
                assert g0 <= g1
                assert o == off and n == int(counts[g0:g1].sum())
                off += n
                # a cut is the genstep boundary nearest its equal-share target
                assert abs(o - total * p / parts) <= counts.max() / 2 + 1
            assert off == total


def test_genstep_slices_edges():
    assert shard.genstep_slices([], 2) == [(0, 0, 0, 0), (0, 0, 0, 0)]
    assert shard.genstep_slices([10], 3) == [(0, 0, 0, 0), (0, 1, 0, 10), (1, 1, 10, 0)]
    assert shard.genstep_slices([0, 0, 6, 0], 2) == [(0, 2, 0, 0), (2, 4, 0, 6)]
    with pytest.raises(ValueError):
        shard.genstep_slices([1, 2], 0)


def test_event_assignment_lpt():
    rng = np.random.default_rng(5)
    c = np.clip(rng.lognormal(np.log(50000), 1.0, size=4096), 1e3, 5e6).astype(np.int64)
    for parts in (1, 2, 4, 8):
        a = shard.event_assignment(c, parts)
        flat = sorted(e for r in a for e in r)
        assert flat == list(range(len(c)))
        loads = [int(c[r].sum()) for r in a]
        assert max(loads) <= c.sum() / parts + c.max()
        assert all(r == sorted(r) for r in a)
    assert shard.event_assignment([], 3) == [[], [], []]
    assert shard.event_assignment([5, 5, 5], 2) == [[0, 2], [1]]


def _scene():
    from opticks_b200 import scenes
    fd, lib, icdf = scenes.detector()
    phys = lib.arrays()
    phys["icdf"] = icdf
    gs = scenes.detector_gensteps(7, 300, seed=9, lib=lib)
    gs.view(np.int32)[:, 0, 3] = [300, 120, 500, 50, 410, 300, 220]   # ragged slices
    return fd, phys, gs


def _oracle_slice_fn(S, u_full):
    """oracle stand-in for one rank's CUDA slice: the slice's uniforms are the rows of its absolute
    photon indices, and sphoton.index is made absolute as photon_offset does on the device"""
    import torch

    def fn(gs_slice, event, off, n):
        photon, seq, err = S.simulate(gs_slice, u_full[off:off + n], 0)
        assert err == 0
        photon.view(np.uint32)[:, 3, 2] += np.uint32(off)
        flags = photon.view(np.uint32)[:, 3, 3]
        hit = photon[(flags & SD) == SD]
        ident = hit.view(np.uint32)[:, 3, 1] & 0xffffff
        sens = np.bincount(ident[ident > 0] - 1, minlength=17612).astype(np.int32)
        return {"photon": torch.from_numpy(photon), "seq": torch.from_numpy(seq.view(np.int64)),
                "hit": torch.from_numpy(hit), "sensor_hits": torch.from_numpy(sens)}

    return fn


def _rank_main(rank, world, port, outdir):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        from oracle import oracle as O
        fd, phys, gs = _scene()
        S = O.Scene(fd.arrays(), phys)
        N = int(shard.genstep_counts(gs).sum())
        u = np.random.default_rng(11).random((N, 256), dtype=np.float32)
        res = shard.simulate_sharded(_oracle_slice_fn(S, u), gs, 0)
        g = shard.gather_rows(torch.arange(rank * 3, dtype=torch.int64).reshape(-1, 1))
        np.savez(os.path.join(outdir, f"rank{rank}.npz"), photon=res["photon"].numpy(), seq=res["seq"].numpy(),
                 hit=res["hit"].numpy(), sensor=res["sensor_hits"].numpy(), sl=np.array(res["slice"]), ragged=g.numpy())
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_gloo_sharded_event_equals_single(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True, start_method="spawn")
    from oracle import oracle as O
    fd, phys, gs = _scene()
    S = O.Scene(fd.arrays(), phys)
    N = int(shard.genstep_counts(gs).sum())
    u = np.random.default_rng(11).random((N, 256), dtype=np.float32)
    full = _oracle_slice_fn(S, u)(gs, 0, 0, N)
    r = [np.load(os.path.join(tmp_path, f"rank{k}.npz")) for k in range(world)]
    photon = np.concatenate([x["photon"] for x in r])
    seq = np.concatenate([x["seq"] for x in r])
    assert [tuple(x["sl"]) for x in r] == shard.genstep_slices(shard.genstep_counts(gs), world)
    assert np.array_equal(photon.view(np.uint32), full["photon"].numpy().view(np.uint32))
    assert np.array_equal(seq, full["seq"].numpy())
    nh = full["hit"].shape[0]
    assert nh > 0
    for x in r:                                   # every rank holds the whole event's hits, in photon order
        assert np.array_equal(x["hit"].view(np.uint32), full["hit"].numpy().view(np.uint32))
        assert np.array_equal(x["sensor"], full["sensor_hits"].numpy())
        assert np.array_equal(x["ragged"].reshape(-1), np.array([0, 1, 2]))   # rank 0 gave 0 rows, rank 1 three
