"""Benchmark of the photon engine on one B200 (one process per GPU under torchrun).

Headline (`value`): photons/s of the plain form on the full synthetic detector — one event of
10,000,000 scintillation photons from 1,000 gensteps (vertices uniform in r < 17 m, 430/20 nm),
17,612 PMT instances, seqhis recorded, SD hits compacted in photon order — gensteps resident
in HBM, device time from CUDA events on the launch stream.

Also on the line:
  e2e          photons/s through the reference-facing host call (CSGOptiXService.simulate:
               H2D gensteps, D2H hits into pinned buffers), timed per step; e2e_full also returns
               every photon and its seq (about 1 GB per step over PCIe)
  roofline     the simulate launch sequence: algorithmic bytes per photon (48 RNG state + 64 sphoton
               + 32 seq + 64 x hit fraction + 96 / photons per genstep) / its duration vs measured HBM
               (the path is latency-bound ray tracing, far from the HBM roof), with the issue figures
               of the dominant kernel from its ncu capture
  cpu_baseline the CPU oracle (port of the reference's path) on all host threads over a stride
               sample of the same event (200 photons of each of its 1,000 gensteps), and the same
               for the C1 and Cerenkov forms
  forms        C1 (1M torch photons, sphere-in-box) and a Cerenkov event (1M photons from 200
               tracks); batched (4,096 lognormal events in one call; the one-kernel persistent form
               autotuned and replayed as a CUDA graph, and the wavefront form) vs the per-event
               loop, with per-event latency p50/p99; the adjoint (C5) cost and FD table; the CSG scan
               (16,777,216 rays vs the 15-node tree with torus, rays/s)

--impl reference: the reference's CPU implementation of the path on the host cores, on the same
stride sample: its own qsim/CSG headers compiled for the CPU under MOCK_CURAND with small GLM and
plog stand-ins (oracle/_ref, kind: reference); the C restatement (kind: port) only where that
build is absent.
Multi-GPU (`--gpus N` re-launches itself under torch.distributed.run when WORLD_SIZE is unset):
each rank simulates its own events (no data-path collective); value = photons of all ranks / max
over ranks of the device time.  A second line item, `sharded`, splits one C3 event across the
ranks (genstep slices) and gathers its hits and sensor counts over NCCL.
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "photons/s"
ENGINE_KW = {}          # engine config overrides from the command line (kernel_mode)
PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
# algorithmic bytes of one photon: the reference's 48 B curandStateXORWOW read (the engine's own
# layout reads 24 B of it), the 64 B sphoton and 32 B sseq writes; + 64 B per hit and the genstep
# share are added per workload
BYTES_PER_PHOTON_FIXED = 48 + 64 + 32
SAMPLE_PER_GENSTEP = 30        # CPU sample: this many photons of every genstep of the event
# DRAM bytes (read + write) of all kernels of one simulate call of this 10M-photon event, from a
# one-pass ncu capture of the bench's own launches (profiles/launches_dram_wavefront_detector_10M.md)
DRAM_TRAFFIC = {"bytes_per_call": 12.723e9, "photons": 10_000_000,
                "source": "ncu dram__bytes_read.sum + dram__bytes_write.sum summed over the 12 launches of one "
                          "10M-photon simulate call of this workload (profiles/launches_dram_wavefront_detector_10M.md)"}
# issue figures of the dominant kernel (k_wave_tail, 68 % of the step) from its ncu --set full
# capture (profiles/k_wave_tail_detector_2M_ncu_full.md)
ISSUE = {"kernel": "k_wave_tail", "share_of_step": 0.68, "issue_active": 0.387, "threads_per_warp_inst": 9.71,
         "warps_active": 0.184, "lane_issue_frac": 0.387 * 9.71 / 32,
         "source": "profiles/k_wave_tail_detector_2M_ncu_full.md"}


def load_peaks():
    try:
        with open(PEAKS) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def detector_workload(num_genstep, per_genstep, seed=0):
    from opticks_b200 import scenes
    fd, lib, icdf = scenes.detector()
    phys = lib.arrays()
    phys["icdf"] = icdf
    gs = scenes.detector_gensteps(num_genstep, per_genstep, seed=seed, lib=lib)
    return fd, lib, phys, gs


class Clocks:
    """nvidia-smi sampling around a timed region: the sampler starts before the warm-up (so it is
    running when the region opens), every sample carries its time, and the summary keeps the
    samples taken inside the region (window marked with begin/end)"""
    Q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    PERIOD_MS = 20

    def __init__(self, device):
        self.device = device
        self.p = None
        self.t0 = self.t1 = None
        self.path = os.path.join(tempfile.gettempdir(), f"phx_bench_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-lms", str(self.PERIOD_MS)], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        return self

    def begin(self):
        # the timed region opens once the sampler has written its first row (nvidia-smi can take
        # longer to start than the warm-up steps last); at most 5 s
        deadline = time.time() + 5.0
        while self.p is not None and self.p.poll() is None and time.time() < deadline:
            try:
                self.f.flush()
                if os.path.getsize(self.path) > 0:
                    break
            except OSError:
                pass
            time.sleep(0.02)
        self.t0 = time.time()

    def end(self):
        self.t1 = time.time()

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()
            self.f.close()

    def summary(self):
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines()]
        except Exception:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        rows = [[c.strip() for c in r] for r in rows if len(r) >= 10]

        def when(r):
            try:
                return datetime.datetime.strptime(r[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
            except ValueError:
                return None
        if self.t0 is not None and self.t1 is not None:
            rows = [r for r in rows if when(r) is not None and self.t0 <= when(r) <= self.t1]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        mx = [float(r[3]) for r in rows if r[3].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[6 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows), "period_ms": self.PERIOD_MS}


def stride_sample(gs, per_genstep=SAMPLE_PER_GENSTEP):
    """the CPU sample of an event: every genstep kept, each with at most `per_genstep` photons, so
    the sample spans the event's vertices (and Cerenkov tracks) as the whole event does"""
    g = np.array(gs, dtype=np.float32, copy=True).reshape(-1, 6, 4)
    c = g.view(np.int32)[:, 0, 3]
    c[:] = np.minimum(c, per_genstep)
    return g


def oracle_rate(fd, phys, gs, reps=1, K=512, seed=123):
    """photons/s of the C restatement (all host threads) over the photons of `gs`, numpy uniforms"""
    from oracle import oracle as O
    S = O.Scene(fd.arrays(), phys)
    n = int(gs.view(np.int32)[:, 0, 3].clip(0).sum())
    u = np.random.Generator(np.random.PCG64(seed)).random((n, K), dtype=np.float32)
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        S.simulate(gs, u, 0)
        times.append(time.perf_counter() - t0)
    return n / statistics.mean(times), n, O.lib().oracle_threads(), times


def reference_rate(fd, phys, gs, reps=1):
    """photons/s of the reference's own qsim/CSG path compiled for the CPU (all host threads), or
    None when that build is absent"""
    from oracle import oracle as O
    if not O.have_ref_cpu_sim():
        return None
    times, n, nt = [], 0, 0
    for r in range(reps):
        ph, _, secs, nt = O.ref_simulate_cpu(fd.arrays(), phys, gs, seed=1 + r, outputs=False)
        times.append(secs)
    n = int(gs.view(np.int32)[:, 0, 3].clip(0).sum())
    return n / statistics.mean(times), n, nt, times


def cpu_rate(fd, phys, gs, reps=1):
    """(photons/s, photons, threads, times, kind): the reference's CPU build where it was built,
    else the C restatement"""
    r = reference_rate(fd, phys, gs, reps)
    if r is not None:
        return (*r, "reference")
    return (*oracle_rate(fd, phys, gs, reps), "port")


KIND_NOTE = {"reference": "the reference's qsim/CSG headers compiled for the CPU (MOCK_CURAND: its mt19937_64 "
                          "uniforms and nearest-sample mock textures), closest hit over world-box-culled instances",
             "port": "the C restatement of the path (numpy uniforms); the reference's CPU build is absent"}


def cpu_baseline(fd, phys, gs, form_workloads=()):
    """the CPU implementation on all host threads over the stride sample of the event (and of each
    form); the C restatement's figure on the same sample beside it"""
    sample = stride_sample(gs)
    v, n, cores, times, kind = cpu_rate(fd, phys, sample, reps=3)
    out = {"value": v, "unit": METRIC, "cores": cores, "kind": kind,
           "sample": f"{SAMPLE_PER_GENSTEP} photons of each of the {len(gs)} gensteps of the event ({n} photons), "
                     f"{KIND_NOTE[kind]}; {len(times)} timed passes of {statistics.mean(times):.1f} s"}
    if kind == "reference":
        pv, _, _, pt = oracle_rate(fd, phys, sample, reps=2)
        out["port"] = {"value": pv, "unit": METRIC, "note": "the C restatement (oracle) on the same sample"}
    forms = {}
    for name, (ffd, fphys, fgs, per, reps) in form_workloads:
        fv, fn, _, ft, fk = cpu_rate(ffd, fphys, stride_sample(fgs, per), reps=reps)
        forms[name] = {"value": fv, "unit": METRIC, "kind": fk, "sample_photons": fn, "passes": reps, "seconds": sum(ft),
                       "sample": f"at most {per} photons of each of the {len(fgs)} gensteps"}
    if forms:
        out["forms"] = forms
    return out


def run_reference(args):
    """--impl reference : CPU implementation of the path on the host cores (rank 0 only), each
    step the stride sample of the C3 event: the reference's own qsim/CSG path compiled for the
    CPU where it was built, else the C restatement"""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    fd, lib, phys, gs = detector_workload(args.gensteps, args.per_genstep)
    sample = stride_sample(gs)
    n = int(sample.view(np.int32)[:, 0, 3].sum())
    for _ in range(args.warmup):
        cpu_rate(fd, phys, stride_sample(gs, 2), reps=1)
    times = []
    kind, cores = "port", 0
    for _ in range(args.steps):
        v1, _, cores, t1, kind = cpu_rate(fd, phys, sample, reps=1)
        times.append(t1[0])
    v = n / statistics.mean(times)
    line = {"metric": METRIC, "value": v, "unit": METRIC, "impl": "reference", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(times), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "detector-17612pmt-scint-10M", "gensteps": args.gensteps,
                       "photons_per_genstep": args.per_genstep, "sample_photons_per_step": n},
            "cpu_baseline": {"value": v, "unit": METRIC, "cores": cores, "kind": kind,
                             "sample": f"{SAMPLE_PER_GENSTEP} photons of each of the {len(gs)} gensteps of the event per "
                                       f"step ({n} photons), {KIND_NOTE[kind]}; warm-up steps take 2 photons per genstep"},
            "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def measure_batched(torch, E, fd, lib, phys, dev, num_event=4096, tune_cache=None):
    """C4: uneven events in one batched call vs the per-event loop, each in both loop forms (the
    one-kernel persistent launch, autotuned and replayed as a CUDA graph, and the wavefront rounds);
    the speed-up compares the faster batched form with the faster per-event loop"""
    from opticks_b200 import autotune, scenes
    gs = scenes.batched_events(num_event, lib=lib)
    ev = np.arange(len(gs), dtype=np.int32)
    counts = gs.view(np.int32)[:, 0, 3].astype(np.int64)
    N = int(counts.sum())
    g = torch.from_numpy(gs).to(dev)
    e = torch.from_numpy(ev).to(dev)
    photon = torch.empty((N, 4, 4), dtype=torch.float32, device=dev)
    seq = torch.empty((N, 2, 2), dtype=torch.int64, device=dev)
    hit = torch.empty((N, 4, 4), dtype=torch.float32, device=dev)
    done = torch.zeros((num_event + 1,), dtype=torch.int64, device=dev)
    st = torch.cuda.current_stream(dev)
    assert st.cuda_stream != 0, "run on a non-default stream so the library launches where the events are recorded"
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    off = np.concatenate([[0], np.cumsum(counts)])
    forms = {}
    for mode in (1, 2):
        eng = E.Engine(fd.arrays(), phys, E.default_config(max_photon=int(counts.max()), num_sensor=scenes.NUM_PMT,
                                                           kernel_mode=mode), device=dev.index)
        if mode == 1:
            best = autotune.tune_batched(eng, gs, ev, torch, cache=tune_cache)
            kw = {k: best[k] for k in ("block", "regroup", "chunk")}
        else:
            best = autotune.tune_wavefront(eng, gs, ev, torch, cache=tune_cache, seq=seq)   # left set on the engine
            kw = {}

        def batch():
            return eng.simulate_batched_device(g, e, N, photon=photon, seq=seq, hit=hit, hit_capacity=N, num_event=num_event,
                                               event_done_ns=done, stream=st.cuda_stream, **kw)
        batch()                      # warm-up (+ graph capture in the persistent form)
        torch.cuda.synchronize()
        e0.record(st)
        nh_b, st_b = batch()
        graph_b = eng.last_call_stats()["graph"]
        e1.record(st)
        torch.cuda.synchronize()
        ms_b = e0.elapsed_time(e1)
        d = done.cpu().numpy()
        lat_b = (d[:num_event] - d[num_event]) / 1e6    # ms from launch start to each event's last photon

        def loop(record=None):
            for k in range(num_event):
                t0 = time.perf_counter()
                eng.simulate_device(g[k:k + 1], int(counts[k]), k, photon=photon[off[k]:off[k + 1]], seq=seq[off[k]:off[k + 1]],
                                    hit=hit[off[k]:off[k + 1]], hit_capacity=int(counts[k]), stream=st.cuda_stream)
                if record is not None:
                    record.append(time.perf_counter() - t0)
        loop()                       # warm-up
        torch.cuda.synchronize()
        per = []
        e0.record(st)
        loop(per)
        e1.record(st)
        torch.cuda.synchronize()
        ms_l = e0.elapsed_time(e1)
        per = np.array(per) * 1e3
        lat_l = np.cumsum(per)
        bounded = None
        if mode == 2:
            # events finishing before the end of the call: a pool of 2^24 paths refilled from the
            # queue (host-read schedule), per-event completion times from the device clock
            eng.set_launch_config(wave_pool=1 << 24, wave_rounds=0)
            batch()
            torch.cuda.synchronize()
            e0.record(st)
            batch()
            e1.record(st)
            torch.cuda.synchronize()
            d = done.cpu().numpy()
            lat_p = (d[:num_event] - d[num_event]) / 1e6
            bounded = {"wave_pool": 1 << 24, "batched_ms": e0.elapsed_time(e1),
                       "event_done_ms_p50_p99": [float(np.percentile(lat_p, 50)), float(np.percentile(lat_p, 99))]}
        eng.close()
        forms["persistent" if mode == 1 else "wavefront"] = {
            "batched_photons_per_s": N / (ms_b / 1e3), "batched_ms": ms_b,
            "loop_photons_per_s": N / (ms_l / 1e3), "loop_ms": ms_l,
            "batched_event_done_ms_p50_p99": [float(np.percentile(lat_b, 50)), float(np.percentile(lat_b, 99))],
            "loop_event_ms_p50_p99": [float(np.percentile(per, 50)), float(np.percentile(per, 99))],
            "loop_event_done_ms_p50_p99": [float(np.percentile(lat_l, 50)), float(np.percentile(lat_l, 99))],
            "cuda_graph": graph_b, "hits": nh_b, "status": st_b,
            "autotuned": {k: best[k] for k in best if k != "table"},
            **({"bounded_pool": bounded} if bounded else {})}
    bb = min(forms, key=lambda k: forms[k]["batched_ms"])
    bl = min(forms, key=lambda k: forms[k]["loop_ms"])
    return {"workload": f"{num_event} events, one scintillation genstep each, lognormal(median 50k, sigma_ln 1) "
                        f"clipped [1e3,5e6], {N} photons",
            "batched_photons_per_s": forms[bb]["batched_photons_per_s"], "batched_form": bb,
            "loop_photons_per_s": forms[bl]["loop_photons_per_s"], "loop_form": bl,
            "speedup_batched_over_loop": forms[bl]["loop_ms"] / forms[bb]["batched_ms"],
            "forms": forms}


def measure_scan(torch, E, dev, n_rays=1 << 24):
    """C2: rays/s of the CSG scan over the 15-node tree with torus (its FP64 distance error is
    measured by the GPU tests against the FP64 oracle)"""
    from opticks_b200 import scenes
    fd, p = scenes.csg_scan_tree(with_torus=True)
    A = fd.arrays()
    _, lib, _, _ = scenes.sphere_in_box(1)
    eng = E.Engine(A, lib.arrays(), E.default_config(max_photon=64), device=dev.index)
    rays = scenes.scan_rays(n_rays, seed=0)
    r = torch.from_numpy(rays).to(dev)
    out = torch.empty((n_rays, 4), dtype=torch.float32, device=dev)
    st = torch.cuda.current_stream(dev)
    assert st.cuda_stream != 0, "run on a non-default stream so the library launches where the events are recorded"
    res = {}
    for pol in (0, 1):
        eng.scan_device(p, r, n_rays, out, 0.0, pol, st.cuda_stream)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(3):
            eng.scan_device(p, r, n_rays, out, 0.0, pol, st.cuda_stream)
        e1.record(st)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / 3
        hits = int((out[:, 3] > 0).sum().item())
        res["polish" if pol else "fp32"] = {"rays_per_s": n_rays / (ms / 1e3), "ms": ms, "hits": hits,
                                            "bytes_per_ray": 40, "achieved_gbs": 40 * n_rays / (ms / 1e3) / 1e9}
    eng.close()
    return dict(workload=f"{n_rays} rays, origins uniform in a 2 m cube, isotropic; 15-node CSG tree with torus", **res)


def measure_plain(torch, E, fd, phys, gs, dev, event=7, reps=5, num_sensor=0):
    """photons/s of one event (device-resident gensteps, photons + seq + hits out), CUDA events on
    the launch stream; status must stay clear (no rejection loop reached its cap)"""
    N = int(gs.view(np.int32)[:, 0, 3].sum())
    eng = E.Engine(fd.arrays(), phys, E.default_config(max_photon=N, num_sensor=num_sensor, **ENGINE_KW), device=dev.index)
    g = torch.from_numpy(gs).to(dev)
    photon = torch.empty((N, 4, 4), dtype=torch.float32, device=dev)
    seq = torch.empty((N, 2, 2), dtype=torch.int64, device=dev)
    hit = torch.empty((N, 4, 4), dtype=torch.float32, device=dev)
    st = torch.cuda.current_stream(dev)
    assert st.cuda_stream != 0
    run = lambda ev: eng.simulate_device(g, N, ev, photon=photon, seq=seq, hit=hit, hit_capacity=N, stream=st.cuda_stream)
    for w in range(3):
        run(event + 1000 + w)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    status, hits = 0, 0
    for r in range(reps):
        nh, stt = run(event + r)
        status |= stt
        hits += nh
    e1.record(st)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    eng.close()
    return {"photons": N, "photons_per_s": N / (ms / 1e3), "ms": ms, "hit_fraction": hits / (N * reps), "status": status,
            "steps": reps}


def c1_workload():
    """C1: 1M torch photons (isotropic, 440 nm, random linear polarisation) in the sphere-in-box"""
    from opticks_b200 import scenes
    fd, lib, _, gs = scenes.sphere_in_box(1_000_000)
    return fd, lib.arrays(), gs


def c1_reference_gs(gs):
    """C1's genstep with the reference's T_SPHERE torch type (its fixed polarisation phase) for the
    CPU baselines: the random-polarisation type is this engine's extension, unknown to the
    reference's storch"""
    from opticks_b200 import scenes
    g = np.array(gs, copy=True)
    g.view(np.int32)[:, 5, 3] = scenes.T_SPHERE
    return g


def cerenkov_workload(lib, num_track=200, per_track=5000, seed=21):
    """1M Cerenkov photons from 200 tracks in the liquid scintillator: 1-40 mm steps, beta from
    0.75 to 0.9999 (the bnd-texture rejection sampling of wavelength and cone angle)"""
    from opticks_b200 import scenes
    rng = np.random.Generator(np.random.PCG64(seed))
    ml = lib.material_line("LS")
    pos = scenes.uniform_ball(num_track, 16000.0, rng)
    gs = []
    for k in range(num_track):
        d = rng.normal(size=3)
        d *= rng.uniform(1.0, 40.0) / np.linalg.norm(d)
        beta = rng.uniform(0.75, 0.9999)
        gs.append(scenes.cerenkov_genstep(per_track, tuple(pos[k]), ml, delta=tuple(d), beta_inverse=1.0 / beta,
                                          time=float(rng.uniform(0.0, 5.0))))
    return np.stack(gs)


def measure_adjoint(torch, E, fd, lib, phys, dev, num_genstep=100, per_genstep=10000, fd_events=4, precise_events=256,
                    rel_step=1e-3, precise_step=1e-3):
    """C5: adjoint pass cost vs the plain forward, and agreement with central finite differences under
    common random numbers (per-parameter means and standard errors over independent events)"""
    from opticks_b200 import adjoint as ADJ
    from opticks_b200 import scenes
    gs = scenes.detector_gensteps(num_genstep, per_genstep, seed=5, lib=lib)
    N = int(gs.view(np.int32)[:, 0, 3].sum())
    mat_line = lib.material_line("LS")
    wl = (300.0, 620.0)
    theta0 = ADJ.nominal_theta(phys, mat_line, *wl)
    eng = E.Engine(fd.arrays(), phys, E.default_config(max_photon=N, num_sensor=scenes.NUM_PMT), device=dev.index)
    g = torch.from_numpy(gs).to(dev)
    hits = torch.zeros((scenes.NUM_PMT,), dtype=torch.float64, device=dev)
    grad = torch.zeros((scenes.NUM_PMT, 32), dtype=torch.float64, device=dev)
    photon = torch.empty((N, 4, 4), dtype=torch.float32, device=dev)
    seq = torch.empty((N, 2, 2), dtype=torch.int64, device=dev)
    hit = torch.empty((N, 4, 4), dtype=torch.float32, device=dev)
    st = torch.cuda.current_stream(dev)
    assert st.cuda_stream != 0

    def timed(fn, reps=5):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(reps):
            fn()
        e1.record(st)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    ms_adj = timed(lambda: ADJ.adjoint_device(eng, g, N, 7, theta0, mat_line, *wl, hits, grad, st.cuda_stream))
    # the score-function estimator alone (every kind's score terms, the Fresnel branch probabilities
    # included), without the refractive index's pathwise tangent
    ms_adj_score = timed(lambda: ADJ.adjoint_device(eng, g, N, 7, theta0, mat_line, *wl, hits, grad, st.cuda_stream,
                                                    pathwise=False))
    ms_fwd = timed(lambda: eng.simulate_device(g, N, 7, photon=photon, seq=seq, hit=hit, hit_capacity=N, stream=st.cuda_stream))
    ms_fwd_bare = timed(lambda: eng.simulate_device(g, N, 7, stream=st.cuda_stream))

    def run(theta, ev):
        ADJ.adjoint_device(eng, g, N, ev, theta.astype(np.float32), mat_line, *wl, hits, grad, st.cuda_stream)
        torch.cuda.synchronize()
        return hits.sum().item(), grad.sum(0).cpu().numpy()

    base = theta0.astype(np.float64)

    def fd_table(params, events, ev0, step):
        """per-event adjoint and CRN central differences for `params`; means and SEs over events"""
        adj = np.zeros((events, 32))
        fdv = np.full((events, 32), np.nan)
        for m in range(events):
            ev = ev0 + m
            _, adj[m] = run(base, ev)
            for k in params:
                h = step * base[k]
                if h <= 0.0:
                    continue           # zero-valued reemission bins: no central difference inside [0, 1]
                tp, tm = base.copy(), base.copy()
                tp[k] += h
                tm[k] -= h
                fdv[m, k] = (run(tp, ev)[0] - run(tm, ev)[0]) / (2 * h)
        rows = []
        for k in params:
            a, f = adj[:, k], fdv[:, k]
            am, ase = float(a.mean()), float(a.std(ddof=1) / np.sqrt(events))
            row = {"k": k, "kind": ADJ.KINDS[k // 8], "bin": k % 8, "theta": float(base[k]), "adjoint": am, "adjoint_se": ase, "fd": None}
            if not np.isnan(f).any():
                fm, fse = float(f.mean()), float(f.std(ddof=1) / np.sqrt(events))
                se = float(np.hypot(ase, fse))
                row.update(fd=fm, fd_se=fse, rel_diff=(am - fm) / fm if fm != 0 else None,
                           z=(am - fm) / se if (se > 0 and fse > 0) else None)
            rows.append(row)
        return rows

    def summary(rows):
        cmp = [r for r in rows if r["fd"] is not None and r.get("z") is not None]
        return {"compared": len(cmp),
                "within_2pct": sum(1 for r in cmp if r["rel_diff"] is not None and abs(r["rel_diff"]) <= 0.02),
                "within_3se": sum(1 for r in cmp if abs(r["z"]) <= 3.0)}

    all_rows = fd_table(range(32), fd_events, 11, rel_step)
    # the bins holding most of the scintillation spectrum (absorption, Rayleigh, refractive index)
    dominant = [2, 3, 4, 10, 11, 26, 27, 28]
    precise = fd_table(dominant, precise_events, 1000, precise_step)
    eng.close()
    return {"workload": f"{N} photons from {num_genstep} scintillation gensteps, theta = 4 properties x 8 bins of LS over 300-620 nm",
            "adjoint_ms": ms_adj, "forward_ms_with_outputs": ms_fwd, "forward_ms_no_outputs": ms_fwd_bare,
            "adjoint_over_forward": ms_adj / ms_fwd, "adjoint_over_forward_no_outputs": ms_adj / ms_fwd_bare,
            "adjoint_score_terms_only_ms": ms_adj_score, "adjoint_score_terms_only_over_forward": ms_adj_score / ms_fwd,
            "adj_wave_rounds": int(eng.config.adj_wave_rounds),
            "fd": {"common_random_numbers": True,
                   "note": "rindex rows include the pathwise refraction term (tangent of the refracted direction "
                           "carried through later segments, Fresnel probabilities and Rayleigh densities; terms "
                           "clipped at 1e4, tangents at 100 per unit n); z is omitted where the CRN difference "
                           "moved no photon in any event",
                   "all_params": {"events": fd_events, "rel_step": rel_step, "summary": summary(all_rows), "rows": all_rows},
                   "dominant_bins": {"events": precise_events, "rel_step": precise_step, "summary": summary(precise),
                                     "rows": precise}}}


def relaunch(n):
    """--gpus N without a launcher: run this script again as N ranks under torch.distributed.run"""
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}", "--master-addr",
           "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__), *sys.argv[1:]]
    sys.exit(subprocess.call(cmd))


def check_ranks():
    """every rank joins a gloo group and sums its rank; rank 0 prints what it saw"""
    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    t = torch.tensor([dist.get_rank()], dtype=torch.int64)
    dist.all_reduce(t)
    if dist.get_rank() == 0:
        print(json.dumps({"check_ranks": dist.get_world_size(), "rank_sum": int(t.item())}), flush=True)
    dist.barrier()
    dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--gensteps", type=int, default=1000)
    ap.add_argument("--per-genstep", type=int, default=10000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true")
    ap.add_argument("--forms", default="c1,cerenkov,batched,scan,adjoint", help="comma list of the forms to measure")
    ap.add_argument("--events", type=int, default=4096)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--kernel-mode", type=int, default=None, help="engine kernel_mode override (1 persistent, 2 wavefront)")
    ap.add_argument("--tune-cache", default=None, help="json file holding the autotuner's choice between runs")
    ap.add_argument("--check-ranks", action="store_true",
                    help="start the ranks and exchange one gloo all-reduce, then exit (launch check, no GPU)")
    args = ap.parse_args()
    if args.kernel_mode is not None:
        ENGINE_KW["kernel_mode"] = args.kernel_mode
    args.warmup = max(args.warmup, 3)
    if "WORLD_SIZE" not in os.environ and args.gpus > 1 and args.impl == "engine":
        return relaunch(args.gpus)
    world_env = int(os.environ.get("WORLD_SIZE", "1"))
    if args.impl == "engine" and world_env != args.gpus:
        sys.exit(f"bench.py: --gpus {args.gpus} but WORLD_SIZE {world_env}")
    if args.check_ranks:
        return check_ranks()
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist
    from opticks_b200 import engine as E
    from opticks_b200 import scenes

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    # a dedicated stream: the library launches on it, and the CUDA events are recorded on it
    work_stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(work_stream)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    fd, lib, phys, gs = detector_workload(args.gensteps, args.per_genstep)
    N = int(gs.view(np.int32)[:, 0, 3].sum())
    eng = E.Engine(fd.arrays(), phys, E.default_config(max_photon=N, num_sensor=scenes.NUM_PMT, **ENGINE_KW), device=local)
    g_dev = torch.from_numpy(gs).to(dev)
    photon = torch.empty((N, 4, 4), dtype=torch.float32, device=dev)
    seq = torch.empty((N, 2, 2), dtype=torch.int64, device=dev)
    hit = torch.empty((N, 4, 4), dtype=torch.float32, device=dev)
    sensor = torch.empty((scenes.NUM_PMT,), dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream

    def step(ev, with_hits=True):
        return eng.simulate_device(g_dev, N, ev, photon=photon, seq=seq, hit=hit if with_hits else None,
                                   hit_capacity=N if with_hits else 0, sensor_hits=sensor if with_hits else None, stream=sp)

    base_event = rank * 1000 + 1          # every rank simulates its own events (event > 0: jumped streams)
    hits_total = 0
    with Clocks(local) as clk:
        for w in range(args.warmup):
            step(base_event + w)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        clk.begin()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        launches = 0
        for s in range(args.steps):
            nh, st = step(base_event + 100 + s)
            hits_total += nh
            launches += eng.last_call_stats()["kernel_launches"]
        e1.record(stream)
        torch.cuda.synchronize()
        clk.end()
        if world > 1:
            dist.barrier()
    ms = e0.elapsed_time(e1)
    ms_max = ms
    mode = int(eng.config.kernel_mode)
    rounds = eng.last_call_stats()["wave_rounds"]
    if world > 1:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_max = float(t.item())
    value = world * N * args.steps / (ms_max / 1e3)

    # dominant kernel alone: the simulate launch without hit selection (genstep scan + jump + kernel)
    k0, k1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ksteps = 3
    k0.record(stream)
    for s in range(ksteps):
        step(base_event + 200 + s, with_hits=False)
    k1.record(stream)
    torch.cuda.synchronize()
    k_ms = k0.elapsed_time(k1) / ksteps
    f_hit = hits_total / (N * args.steps)
    ppg = N / len(gs)
    bytes_per_photon = BYTES_PER_PHOTON_FIXED + 64.0 * f_hit + 96.0 / ppg
    peak, peak_kind = load_peaks()
    achieved = N * bytes_per_photon / (k_ms / 1e3) / 1e9

    # end to end through the host API with pinned buffers.  e2e: the reference-facing service call
    # (CSGOptiXService.simulate: gensteps in, hits out); e2e_full: photons + seq + hits returned
    ph_h = torch.empty((N, 4, 4), dtype=torch.float32, pin_memory=True).numpy()
    sq_h = torch.empty((N, 2, 2), dtype=torch.int64, pin_memory=True).numpy().view(np.uint64)
    ht_h = torch.empty((N, 4, 4), dtype=torch.float32, pin_memory=True).numpy()
    gs_h = torch.from_numpy(gs).pin_memory().numpy()

    def host_run(full, ev0):
        times, d2h = [], []
        for s in range(args.e2e_steps + 1):
            t0 = time.perf_counter()
            out = eng.simulate_into(gs_h, ev0 + s, ph_h if full else None, sq_h if full else None, ht_h)
            dt = time.perf_counter() - t0
            if s > 0:
                times.append(dt)
                d2h.append((N * 96 if full else 0) + out["num_hit"] * 64)
        return {"value": N / statistics.mean(times), "unit": METRIC, "h2d_bytes_per_step": int(gs.nbytes),
                "d2h_bytes_per_step": int(statistics.mean(d2h)), "ms_per_step": 1e3 * statistics.mean(times)}
    e2e = dict(host_run(False, base_event + 300), api="phx_simulate: host gensteps in, host hits out (CSGOptiXService.simulate)")
    e2e_full = dict(host_run(True, base_event + 400), api="phx_simulate: host gensteps in, host photons + seq + hits out")
    sharded = None
    if world > 1:
        # strong scaling: one C3 event split across the ranks in genstep slices (photon offsets keep
        # the single-GPU RNG streams), hits all-gathered in photon order and sensor counts summed
        from opticks_b200 import shard
        fn = shard.engine_slice_fn(eng, dev, num_sensor=scenes.NUM_PMT, stream=sp)
        shard.simulate_sharded(fn, gs, 1)
        torch.cuda.synchronize()
        dist.barrier()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = 3
        s0.record(stream)
        for r in range(reps):
            out = shard.simulate_sharded(fn, gs, 2 + r)
        s1.record(stream)
        torch.cuda.synchronize()
        t = torch.tensor([s0.elapsed_time(s1) / reps], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        sharded = {"photons_per_s": N / (float(t.item()) / 1e3), "ms_per_event": float(t.item()), "photons_per_event": N,
                   "hits_gathered": int(out["hit"].shape[0]), "scaling": "strong",
                   "note": "one event split across the ranks (genstep slices), NCCL all-gather of hits and all-reduce "
                           "of per-sensor counts inside the timed region; max over ranks"}
        del out
    eng.close()
    del photon, seq, hit
    torch.cuda.empty_cache()

    clocks = clk.summary()
    if rank == 0:
        forms = None
        c1_fd, c1_phys, c1_gs = c1_workload()
        ck_gs = cerenkov_workload(lib)
        if not args.no_forms and world == 1:
            runners = {
                "c1": lambda: dict(measure_plain(torch, E, c1_fd, c1_phys, c1_gs, dev),
                                   workload="C1: 1,000,000 torch photons (T_SPHERE with random linear polarisation, 440 nm) "
                                            "from the centre of a 1 m water sphere in a 3 m detecting box"),
                "cerenkov": lambda: dict(measure_plain(torch, E, fd, phys, ck_gs, dev, num_sensor=scenes.NUM_PMT),
                                         workload=f"detector, {len(ck_gs)} Cerenkov tracks x 5,000 photons, beta 0.75-0.9999, "
                                                  "1-40 mm steps in the liquid scintillator"),
                "batched": lambda: measure_batched(torch, E, fd, lib, phys, dev, args.events, tune_cache=args.tune_cache),
                "scan": lambda: measure_scan(torch, E, dev),
                "adjoint": lambda: measure_adjoint(torch, E, fd, lib, phys, dev)}
            forms = {k: runners[k]() for k in args.forms.split(",") if k}
        cpu = None if args.no_cpu_baseline or world > 1 else cpu_baseline(
            fd, phys, gs, form_workloads=(("c1", (c1_fd, c1_phys, c1_reference_gs(c1_gs), 200_000, 10)),
                                          ("cerenkov", (fd, phys, ck_gs, 100, 1))))
        line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": "detector-17612pmt-scint-10M", "gensteps": len(gs), "photons_per_genstep": int(ppg),
                           "photons_per_step": N, "outputs": "photon+seq+hits(SD)+sensor counts",
                           "l2": "inputs larger than L2 (RNG states 240 MB read + 960 MB written per step)",
                           "kernel": (f"wavefront: closest-hit and physics kernels over every photon of the event "
                                      f"in flight, {rounds} rounds per step, then the tail kernel" if mode == 2 else
                                      "persistent work queue, block 64, refill every bounce"),
                           "parallelism": f"{world} independent event streams" if world > 1 else "1 GPU"},
                "gpu_launches": launches,
                "hit_fraction": f_hit,
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                             "traffic": DRAM_TRAFFIC["bytes_per_call"] * N / DRAM_TRAFFIC["photons"] if mode == 2 else None,
                             "traffic_source": DRAM_TRAFFIC["source"] if mode == 2 else None,
                             "issue": ISSUE if mode == 2 else None,
                             "kernel_ms": k_ms,
                             "kernel": ("k_wave_init + 2 k_wave_trace_df/k_wave_shade rounds + k_wave_tail (whole simulate launch sequence)"
                                        if mode == 2 else "k_sim_persistent (whole simulate launch sequence)"),
                             "bytes_per_photon": bytes_per_photon, "peak_kind": f"{peak_kind} hbm_gbs",
                             "note": "issue/latency-bound divergent ray tracing + physics; HBM roof far from binding"},
                "e2e": e2e, "e2e_full": e2e_full, "clocks": clocks, "cpu_baseline": cpu, "forms": forms,
                "sharded": sharded}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
