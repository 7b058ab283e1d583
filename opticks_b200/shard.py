"""The photon path on several GPUs: one process per GPU, torch.distributed for the plumbing.

Photons are independent given (genstep, absolute photon index, event index): a photon's RNG slot
is its absolute index in the event and the event jump is applied per event.  So an event split
into contiguous genstep slices, each simulated with photon_offset = the slice's first photon,
reproduces the single-GPU photons, seq and hits exactly.  This is the reference's genstep slicing
of large events (qudarap/QSim.cc:436-595: one launch per slice, params.photon_slot_offset,
CSGOptiX/CSGOptiX7.cu:441) with the slices placed on different GPUs instead of run in sequence.
Many small events are instead dealt out whole (longest first, to the least-loaded rank), each
rank running its share as one batched launch.

There is no exchange inside the bounce loop.  The collectives come after the simulation:
  hits         all_gather of the variable-length hit arrays, concatenated in rank order, which is
               photon order because the slices are contiguous and in rank order
  sensor hits  all_reduce (sum) of the per-sensor counts
  adjoint      all_reduce (sum) of H (num_sensor) and J (num_sensor, 32)
"""
from __future__ import annotations

import numpy as np


def genstep_counts(gs: np.ndarray) -> np.ndarray:
    """photon count per genstep (quad6 q0.w as int32), negative counts as 0"""
    g = np.ascontiguousarray(gs, np.float32).reshape(-1, 6, 4)
    return np.maximum(g.view(np.int32)[:, 0, 3].astype(np.int64), 0)


def genstep_slices(counts, parts: int) -> list[tuple[int, int, int, int]]:
    """Split gensteps into `parts` contiguous slices balanced by photon count.

    Returns (g0, g1, photon_offset, num_photon) per part: gensteps [g0, g1) holding photons
    [photon_offset, photon_offset + num_photon).  Cuts fall on genstep boundaries (a genstep is
    never split), at the boundary nearest each equal-share target; slices may be empty when there
    are fewer gensteps than parts."""
    if parts < 1:
        raise ValueError("parts must be >= 1")
    counts = np.asarray(counts, np.int64).reshape(-1)
    G = len(counts)
    cum = np.concatenate([[0], np.cumsum(counts)])
    total = int(cum[-1])
    cuts = [0]
    for p in range(1, parts):
        target = total * p / parts
        j = int(np.searchsorted(cum, target))          # first boundary with cum >= target
        j = min(max(j, 0), G)
        if j > 0 and abs(cum[j - 1] - target) <= abs(cum[j] - target):
            j -= 1
        cuts.append(max(j, cuts[-1]))
    cuts.append(G)
    return [(cuts[p], cuts[p + 1], int(cum[cuts[p]]), int(cum[cuts[p + 1]] - cum[cuts[p]])) for p in range(parts)]


def event_assignment(event_counts, parts: int) -> list[list[int]]:
    """Deal whole events to `parts` ranks, longest first to the least-loaded rank (ties: lowest
    rank, then lowest event index).  Each rank's list is in ascending event order.  The largest
    per-rank load is at most the mean load plus the largest event."""
    if parts < 1:
        raise ValueError("parts must be >= 1")
    c = np.asarray(event_counts, np.int64).reshape(-1)
    order = sorted(range(len(c)), key=lambda e: (-int(c[e]), e))
    load = [0] * parts
    out: list[list[int]] = [[] for _ in range(parts)]
    for e in order:
        r = min(range(parts), key=lambda q: (load[q], q))
        out[r].append(e)
        load[r] += int(c[e])
    return [sorted(x) for x in out]


def _dist():
    import torch.distributed as dist
    return dist


def rank_world(group=None) -> tuple[int, int]:
    dist = _dist()
    if not (dist.is_available() and dist.is_initialized()):
        return 0, 1
    return dist.get_rank(group), dist.get_world_size(group)


def gather_rows(t, group=None):
    """all_gather of a tensor whose leading dimension differs per rank; returns the rank-order
    concatenation on every rank (works for gloo on CPU tensors and NCCL on CUDA tensors)"""
    import torch
    dist = _dist()
    rank, world = rank_world(group)
    if world == 1:
        return t
    n = torch.tensor([t.shape[0]], dtype=torch.int64, device=t.device)
    sizes = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(sizes, n, group=group)
    sizes = [int(s.item()) for s in sizes]
    m = max(sizes)
    pad = torch.zeros((m,) + tuple(t.shape[1:]), dtype=t.dtype, device=t.device)
    if t.shape[0]:
        pad[: t.shape[0]] = t
    bufs = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(bufs, pad, group=group)
    return torch.cat([b[:s] for b, s in zip(bufs, sizes)], dim=0)


def allreduce_sum_(t, group=None):
    """in-place sum over ranks"""
    dist = _dist()
    _, world = rank_world(group)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t


def simulate_sharded(slice_fn, gs: np.ndarray, event: int = 0, group=None, gather_hits: bool = True) -> dict:
    """Simulate one event split across the ranks of `group`.

    slice_fn(gs_slice, event, photon_offset, num_photon) -> dict of tensors for that slice:
    "photon" (n,4,4), "seq" (n,2,2), "hit" (h,4,4) and optionally "sensor_hits" (num_sensor,) int32.
    Returns this rank's slice (photon, seq), its bounds, the hits of the whole event on every rank
    (photon order) and the summed per-sensor counts."""
    rank, world = rank_world(group)
    gs = np.ascontiguousarray(gs, np.float32).reshape(-1, 6, 4)
    sl = genstep_slices(genstep_counts(gs), world)
    g0, g1, off, n = sl[rank]
    out = slice_fn(gs[g0:g1], event, off, n)
    res = {"slice": (g0, g1, off, n), "slices": sl, "photon": out.get("photon"), "seq": out.get("seq")}
    if gather_hits and out.get("hit") is not None:
        res["hit"] = gather_rows(out["hit"], group)
    if out.get("sensor_hits") is not None:
        res["sensor_hits"] = allreduce_sum_(out["sensor_hits"], group)
    return res


def engine_slice_fn(engine, device, num_sensor: int = 0, stream=None):
    """slice_fn running the CUDA engine on `device` (torch CUDA tensors out)"""
    import torch

    def fn(gs_slice, event, photon_offset, num_photon):
        n = int(num_photon)
        photon = torch.empty((n, 4, 4), dtype=torch.float32, device=device)
        seq = torch.empty((n, 2, 2), dtype=torch.int64, device=device)
        hit = torch.empty((n, 4, 4), dtype=torch.float32, device=device)
        sens = torch.zeros((num_sensor,), dtype=torch.int32, device=device) if num_sensor else None
        nh = 0
        if n:
            g = torch.from_numpy(np.ascontiguousarray(gs_slice, np.float32)).to(device)
            s = stream if stream is not None else torch.cuda.current_stream(device).cuda_stream
            nh, status = engine.simulate_device(g, n, event, photon=photon, seq=seq, hit=hit, hit_capacity=n,
                                                sensor_hits=sens, stream=s, photon_offset=int(photon_offset))
            if status:
                raise RuntimeError(f"phx_simulate_device status 0x{status:x}")
        return {"photon": photon, "seq": seq, "hit": hit[:nh], "sensor_hits": sens}

    return fn


def adjoint_sharded(engine, gs: np.ndarray, events, theta, mat_line: int, wl_lo: float, wl_hi: float,
                    device, group=None):
    """Mean over `events` of the expected-hits estimator H (num_sensor) and of J = dH/dtheta
    (num_sensor, 32), the events dealt out across the ranks and the sums all-reduced, so every
    rank returns the same (H, J).  Each event is simulated whole on one GPU."""
    import torch
    from . import adjoint as ADJ
    rank, world = rank_world(group)
    events = [int(e) for e in events]
    if not events:
        raise ValueError("no events")
    n = int(genstep_counts(gs).sum())
    mine = event_assignment([n] * len(events), world)[rank]
    ns = engine.num_sensor
    hits = torch.zeros((ns,), dtype=torch.float64, device=device)
    grad = torch.zeros((ns, 32), dtype=torch.float64, device=device)
    h1 = torch.empty_like(hits)
    j1 = torch.empty_like(grad)
    g = torch.from_numpy(np.ascontiguousarray(gs, np.float32).reshape(-1, 6, 4)).to(device)
    st = torch.cuda.current_stream(device).cuda_stream
    for i in mine:
        ADJ.adjoint_device(engine, g, n, events[i], theta, mat_line, wl_lo, wl_hi, h1, j1, st)
        hits += h1
        grad += j1
    allreduce_sum_(hits, group)
    allreduce_sum_(grad, group)
    return hits / len(events), grad / len(events)
