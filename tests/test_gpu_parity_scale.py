"""Parity at the benchmark configurations' sizes and on the surface branches.

* the surface branch of qsim::propagate_at_surface (qudarap/qsim.h:1680-1750): detect, absorb,
  diffuse (Lambertian, :1988-2020 with the Marsaglia loop :433-575) and specular (:2022-2093)
  reflection on the walls of the sphere-in-box, 200k photons each, against the reference's own
  device code on the same cuRAND streams;
* the zplus_sensor_A surface kind and the lposcost < 0 branch of qsim::propagate (:2304-2316,
  propagate_at_surface_Detect :1753) on the detector with a reflecting rock wall, so photons come
  back onto the backs of the PMTs;
* the full C1 configuration (1,000,000 torch photons) and a 200k-photon sample of the C3 event
  (20 of its 1,000 gensteps, spread over it), the latter also through a small wavefront pool so
  the refill rounds and the tail kernel run under the comparison;
* the FP64 intersection-distance error of C1's and C3's geometry (engine trace vs the FP64 CSG
  oracle along the same rays).

Bar: seqhis identical for >= 99.9 % of photons, position/time/direction/polarisation within 1e-4
relative for >= 99.9 % of those."""
import collections

import numpy as np
import pytest

from oracle import oracle as O
from opticks_b200 import material as M
from opticks_b200 import scenes
from tests._parity import describe, frac_close, seq_match

pytestmark = pytest.mark.gpu

SEQ_BAR = 0.999
TOL = 1e-4
NEED_REF = pytest.mark.skipif(not O.have_ref_sim(), reason="reference GPU build absent")


def _engine(fd, phys, **cfg):
    from opticks_b200 import engine as E
    return E.Engine(fd.arrays(), phys, E.default_config(**cfg))


def _points(seq):
    """number of recorded points (nonzero seqhis nibbles) per photon"""
    s = seq[:, 0, :]
    n = np.zeros(len(s), np.int64)
    for w in range(2):
        for k in range(16):
            n += (((s[:, w] >> np.uint64(4 * k)) & np.uint64(0xF)) != 0)
    return n


def _compare(name, res, ph, sq, chaotic_after=None):
    """seqhis and photon agreement with the reference's device code; prints the mismatch tally.
    ``chaotic_after``: photons with more recorded points than this are tallied apart (they may
    drift beyond 1e-4: a specular box around a sphere is a dispersing billiard, where a last-bit
    difference of one reflection grows by the sphere's focusing factor at every later one); the
    1e-4 bar applies to the rest, and the long chains must still agree in seqhis"""
    from opticks_b200 import engine as E
    m = seq_match(res["seq"], sq)
    same = np.all(res["seq"][:, 0, :] == sq[:, 0, :], axis=1)
    ndiff = int((~same).sum())
    if chaotic_after is not None:
        npt = _points(sq)
        longc = npt > chaotic_after
        fc_long = frac_close(res["photon"], ph, same & longc, TOL)
        print(f"{name}: {int(longc.sum())} photons with > {chaotic_after} points, within 1e-4 {fc_long:.6f}; by points:",
              {int(k): round(frac_close(res["photon"], ph, same & (npt == k), TOL), 5) for k in np.unique(npt) if k >= 8})
        same = same & ~longc
    fc = frac_close(res["photon"], ph, same, TOL)
    bad = collections.Counter(E.seqhis_label(int(a[0, 0]), int(a[0, 1])) + "  |ref: " + E.seqhis_label(int(b[0, 0]), int(b[0, 1]))
                              for a, b in zip(res["seq"][~same][:5], sq[~same][:5]))
    print(f"{name}: {len(sq)} photons, seqhis match {m:.6f} ({ndiff} differ), within 1e-4 {fc:.6f} "
          f"({describe(res['photon'], ph, same, TOL)}); first differing: {dict(bad)}")
    assert m >= SEQ_BAR
    assert fc >= SEQ_BAR
    np.testing.assert_array_equal(res["seq"][same, 1, :], sq[same, 1, :])    # seqbnd
    return same


def _nibble_count(seq, nib):
    """photons whose seqhis holds the given flag nibble at least once"""
    s = seq[:, 0, :]
    hit = np.zeros(len(s), bool)
    for w in range(2):
        for k in range(16):
            hit |= ((s[:, w] >> np.uint64(4 * k)) & np.uint64(0xF)) == np.uint64(nib)
    return int(hit.sum())


# ---------------------------------------------------------------- surface branches
SURFACE_CASES = {
    "mixed": dict(detect=0.2, absorb=0.2, reflect_specular=0.3, reflect_diffuse=0.3),
    "diffuse": dict(detect=0.1, absorb=0.2, reflect_specular=0.0, reflect_diffuse=0.7),
    "specular": dict(detect=0.1, absorb=0.2, reflect_specular=0.7, reflect_diffuse=0.0),
}


@NEED_REF
@pytest.mark.parametrize("case", list(SURFACE_CASES))
def test_surface_reflection_matches_reference(cuda, case):
    from opticks_b200 import engine as E
    n = 200_000
    fd, lib, _, gs = scenes.sphere_in_box_surface(n, **SURFACE_CASES[case])
    phys = lib.arrays()
    eng = _engine(fd, phys, max_photon=n)
    res = eng.simulate(gs, 3)
    eng.close()
    assert res["status"] == 0, E.status_names(res["status"])
    ph, sq = O.ref_simulate_gpu(fd.arrays(), phys, gs, event_index=3)
    _compare(f"surface {case}", res, ph, sq, chaotic_after=12 if SURFACE_CASES[case]["reflect_specular"] > 0 else None)
    ndr, nsr = _nibble_count(res["seq"], 9), _nibble_count(res["seq"], 10)
    print(f"   photons with DR {ndr}, with SR {nsr}, hits {res['num_hit']}")
    c = SURFACE_CASES[case]
    if c["reflect_diffuse"] > 0:
        assert ndr > n // 10
    else:
        assert ndr == 0
    if c["reflect_specular"] > 0:
        assert nsr > n // 10
    else:
        assert nsr == 0


@pytest.mark.parametrize("case", ["mixed", "diffuse"])
def test_surface_reflection_matches_cpu_oracle(cuda, case):
    """the same branches against the C restatement with the engine's uniforms (the Lambertian loop
    draws 3 uniforms per try)"""
    n = 3000
    fd, lib, _, gs = scenes.sphere_in_box_surface(n, **SURFACE_CASES[case])
    phys = lib.arrays()
    eng = _engine(fd, phys, max_photon=n)
    res = eng.simulate(gs, 0)
    u = eng.rng_sequence(0, 0, n, 4096)
    eng.close()
    S = O.Scene(fd.arrays(), phys)
    ph, sq, err = S.simulate(gs, u, 0)
    assert err & 1 == 0
    m = seq_match(res["seq"], sq)
    same = np.all(res["seq"][:, 0, :] == sq[:, 0, :], axis=1)
    short = _points(sq) <= 12
    fc = frac_close(res["photon"], ph, same & short, TOL)
    print(f"surface {case} vs CPU oracle: seqhis {m:.6f} close {fc:.6f} on {int(short.sum())} photons of <= 12 points, "
          f"{frac_close(res['photon'], ph, same & ~short, TOL):.6f} on the longer chains")
    assert m >= 0.995
    # IEEE libm against fast-math intrinsics: each diffuse reflection renormalises a difference of
    # nearly equal vectors (the facet normal), so the ulp differences grow along the chain; the
    # longer chains are tallied, not failed
    assert fc >= 0.995


# ---------------------------------------------------------------- zplus sensor A + lposcost < 0
ROCK_MIRROR = M.Surface("RockMirror", detect=0.0, absorb=0.3, reflect_specular=0.4, reflect_diffuse=0.3)


def _local_cost(fd_arrays, photon):
    """cosine of the polar angle of each photon's end position in its PMT's frame (identity =
    sensor index + 1 = instance index of the PMT)"""
    inst = fd_arrays["inst"].astype(np.float64)
    ident = photon.view(np.uint32)[:, 3, 1] & 0xFFFFFF
    m = inst[ident].copy()
    m[:, :3, 3] = 0.0
    m[:, 3, 3] = 1.0
    inv = np.linalg.inv(m)
    p = np.c_[photon[:, 0, :3].astype(np.float64), np.ones(len(photon))]
    lp = np.einsum("ni,nij->nj", p, inv)[:, :3]
    return lp[:, 2] / np.linalg.norm(lp, axis=1)


@NEED_REF
def test_zplus_sensor_a_matches_reference(cuda):
    from opticks_b200 import engine as E
    fd, lib, icdf = scenes.detector(pmt_ems=M.EMS_SENSOR_A, world_surface=ROCK_MIRROR)
    phys = lib.arrays()
    phys["icdf"] = icdf
    gs = scenes.detector_gensteps(20, 10000, seed=11, lib=lib)
    N = 200_000
    eng = _engine(fd, phys, max_photon=N, num_sensor=scenes.NUM_PMT)
    res = eng.simulate(gs, 2, sensor_hits=True)
    eng.close()
    assert res["status"] == 0, E.status_names(res["status"])
    A = fd.arrays()
    ph, sq = O.ref_simulate_gpu(A, phys, gs, event_index=2)
    p = res["photon"]
    u = p.view(np.uint32)
    # Photons ending on the flat underside of the PMT cap (the zsphere's z = 0 plane, outside the
    # neck) sit exactly on the lposcost = 0 boundary between the two branches: the sign of the
    # local z of the hit is rounding noise of lo.z + t*ld.z, so the branch (always SD, or the
    # detect/absorb draw) is a coin flip between any two builds.  They are the tallied
    # coincident-surface set; the seqhis bar applies to every other photon.
    on_pmt_any = ((u[:, 3, 1] & 0xFFFFFF) > 0) & ((u[:, 3, 0] & 0xFFFF) != 0)
    lc_all = np.ones(len(p))
    lc_all[on_pmt_any] = _local_cost(A, p[on_pmt_any])
    plane = on_pmt_any & (np.abs(lc_all) < 1e-3)
    same = np.all(res["seq"][:, 0, :] == sq[:, 0, :], axis=1)
    print(f"   lposcost = 0 plane: {int(plane.sum())} photons end there, {int((~same & plane).sum())} of them differ; "
          f"{int((~same & ~plane).sum())} differ elsewhere")
    keep = ~plane
    _compare("zplus_sensor_A detector (off the lposcost = 0 plane)", {k: (v[keep] if k in ("seq", "photon") else v)
                                                                     for k, v in res.items()}, ph[keep], sq[keep])
    # which branch each PMT-ending photon took, from its end point in the PMT frame
    flag = u[:, 3, 0] & 0xFFFF                     # orient_boundary_flag: last flag low 16 bits
    bnd = (u[:, 3, 0] >> 16) & 0x7FFF
    b_pmt = lib.boundaries.index(("Water", "PMTCathode", "PMTCathode", "Pyrex"))
    on_pmt = (bnd == b_pmt) & ((flag == 0x40) | (flag == 0x80)) & ((u[:, 3, 1] & 0xFFFFFF) > 0)
    lc = _local_cost(A, p[on_pmt])
    fl = flag[on_pmt]
    front, back = lc > 1e-3, lc < -1e-3
    print(f"   PMT ends: front {int(front.sum())} (SD {int((fl[front] == 0x40).sum())}), "
          f"back {int(back.sum())} (SD {int((fl[back] == 0x40).sum())}, SA {int((fl[back] == 0x80).sum())})")
    assert front.sum() > 1000 and np.all(fl[front] == 0x40)          # propagate_at_surface_Detect: always SD
    assert back.sum() > 100 and (fl[back] == 0x80).sum() > 0 and (fl[back] == 0x40).sum() > 0
    assert _nibble_count(res["seq"], 9) > 100 and _nibble_count(res["seq"], 10) > 100   # rock DR / SR


# ---------------------------------------------------------------- full C1
@NEED_REF
def test_c1_full_config_matches_reference(cuda):
    from opticks_b200 import engine as E
    n = 1_000_000
    fd, lib, _, _ = scenes.sphere_in_box(n)
    gs = scenes.torch_genstep(n, wavelength=440.0, radius=0.0, type_=scenes.T_SPHERE, distance=0.25)[None]
    phys = lib.arrays()
    eng = _engine(fd, phys, max_photon=n)
    res = eng.simulate(gs, 0)
    eng.close()
    assert res["status"] == 0, E.status_names(res["status"])
    ph, sq = O.ref_simulate_gpu(fd.arrays(), phys, gs)
    _compare("C1 1M", res, ph, sq)


# ---------------------------------------------------------------- C3 sample
@pytest.fixture(scope="module")
def c3_sample(cuda):
    """20 of the 1,000 gensteps of the C3 event (every 50th), 200k photons, and the reference's run"""
    fd, lib, icdf = scenes.detector()
    phys = lib.arrays()
    phys["icdf"] = icdf
    gs_all = scenes.detector_gensteps(1000, 10000, seed=0, lib=lib)
    gs = np.ascontiguousarray(gs_all[::50])
    ph, sq = O.ref_simulate_gpu(fd.arrays(), phys, gs, event_index=1) if O.have_ref_sim() else (None, None)
    return dict(fd=fd, lib=lib, phys=phys, gs=gs, ref=(ph, sq))


@NEED_REF
@pytest.mark.parametrize("pool", [0, 1 << 14])
def test_c3_sample_matches_reference(c3_sample, pool):
    """default pool (every photon in flight) and a 16,384-slot pool (the queue refills the pool for
    ~12 rounds and the tail kernel finishes the last paths)"""
    from opticks_b200 import engine as E
    fd, phys, gs = c3_sample["fd"], c3_sample["phys"], c3_sample["gs"]
    N = int(gs.view(np.int32)[:, 0, 3].sum())
    assert N == 200_000 and len(gs) == 20
    eng = _engine(fd, phys, max_photon=N, num_sensor=scenes.NUM_PMT, wave_pool=pool)
    res = eng.simulate(gs, 1, sensor_hits=True)
    stats = eng.last_call_stats()
    eng.close()
    assert res["status"] == 0, E.status_names(res["status"])
    print(f"   pool {pool}: {stats['wave_rounds']} wavefront rounds, {stats['kernel_launches']} launches")
    if pool:
        assert stats["wave_rounds"] >= N // pool         # refilled: at least one round per pool of photons
    ph, sq = c3_sample["ref"]
    same = _compare(f"C3 200k sample pool {pool}", res, ph, sq)
    # per-sensor hits: the engine's counts against the reference's photons
    ref_hit = ph.view(np.uint32)[:, 3, 3] & 0x40 == 0x40
    ids = ph.view(np.uint32)[ref_hit, 3, 1] & 0xFFFFFF
    ref_counts = np.bincount(ids - 1, minlength=scenes.NUM_PMT)
    diff = np.abs(ref_counts.astype(np.int64) - res["sensor_hits"].astype(np.int64)).sum()
    print(f"   hits {res['num_hit']} vs reference {int(ref_hit.sum())}, per-sensor |diff| summed {diff}")
    assert diff <= 2 * int((~same).sum()) + 2


# ---------------------------------------------------------------- FP64 distance error
def _fp64_distance_error(fd, lib, rays, tmin=0.05, polish=0):
    """relative distance error of the engine's closest hits along `rays` against the FP64 evaluator
    on the same prim; tmin is the propagate epsilon, as every simulation trace uses"""
    eng = _engine(fd, lib.arrays(), max_photon=64, root_polish=polish)
    prd, st = eng.trace(rays, tmin, 1e6)
    eng.close()
    assert st == 0
    u = prd.view(np.uint32)
    hit = u[:, 1, 3] != 0xFFFFFFFF
    A = fd.arrays()
    inst = (u[hit, 1, 2] >> 16).astype(np.int64)
    gprim = (u[hit, 1, 3] >> 16).astype(np.int64)
    t64 = O.trace_t64(A, rays[:, hit], inst, gprim, tmin)
    t32 = prd[hit, 0, 3].astype(np.float64)
    missed64 = t64 <= 0
    ok = ~missed64
    err = np.abs(t32[ok] - t64[ok])
    # FP32 resolves a world position to ~1e-7 of its coordinates, so the error is relative to the
    # position scale of the ray (its origin's distance from the world origin) or to t if larger
    scale = np.maximum(np.maximum(np.linalg.norm(rays[:3, hit].T.astype(np.float64), axis=1)[ok], t64[ok]), 1.0)
    rel = err / scale
    q = lambda a, f: float(np.quantile(a, f))
    return dict(rays=rays.shape[1], hits=int(hit.sum()), fp64_disagrees=int(missed64.sum()),
                p50=q(rel, 0.5), p99=q(rel, 0.99), p999=q(rel, 0.999), p9999=q(rel, 0.9999), max=float(rel.max()),
                abs_mm_p999=q(err, 0.999), abs_mm_max=float(err.max()))


def _iso_rays(n, rng, origins):
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return np.ascontiguousarray(np.concatenate([origins.T, d.T]).astype(np.float32))


@pytest.mark.parametrize("polish", [0, 1])
def test_c1_fp64_distance_error(cuda, polish):
    """rays from uniform points of the box through the sphere-in-box geometry: the engine's closest
    hit distance against the FP64 evaluator along the same ray to the same prim, without and with
    the FP64 root polish"""
    rng = np.random.default_rng(3)
    n = 1 << 20
    fd, lib, _, _ = scenes.sphere_in_box(1)
    rays = _iso_rays(n, rng, rng.uniform(-1490.0, 1490.0, size=(n, 3)))
    r = _fp64_distance_error(fd, lib, rays, polish=polish)
    print(f"C1 FP64 distance error (polish {polish}): {r}")
    assert r["hits"] == n                      # every ray from inside the box hits something
    assert r["fp64_disagrees"] == 0
    assert r["p999"] < 1e-5


@pytest.mark.parametrize("polish", [0, 1])
def test_c3_fp64_distance_error(cuda, polish):
    """rays from uniform points inside the water sphere of the detector (17,612 PMTs); the relative
    error grows near tangency (grazing PMT caps and necks), which the upper quantiles show"""
    rng = np.random.default_rng(4)
    n = 1 << 20
    fd, lib, _ = scenes.detector()
    rays = _iso_rays(n, rng, scenes.uniform_ball(n, 20400.0, rng))
    r = _fp64_distance_error(fd, lib, rays, polish=polish)
    print(f"C3 FP64 distance error (polish {polish}): {r}")
    assert r["hits"] == n
    assert r["fp64_disagrees"] <= n // 100000
    assert r["p999"] < 1e-5


# ---------------------------------------------------------------- Cerenkov at scale
@NEED_REF
def test_cerenkov_event_matches_reference(cuda):
    """120,000 Cerenkov photons from 40 tracks of beta 0.75-0.9999 in the liquid scintillator (the
    bnd-texture rejection sampling of wavelength and cone angle, qudarap/qcerenkov.h:56-320):
    seqhis and photons against the reference's device code, and no rejection loop at its cap"""
    from opticks_b200 import engine as E
    fd, lib, icdf = scenes.detector()
    phys = lib.arrays()
    phys["icdf"] = icdf
    ml = lib.material_line("LS")
    rng = np.random.Generator(np.random.PCG64(41))
    pos = scenes.uniform_ball(40, 16000.0, rng)
    gs = []
    for k in range(40):
        d = rng.normal(size=3)
        d *= rng.uniform(1.0, 40.0) / np.linalg.norm(d)
        gs.append(scenes.cerenkov_genstep(3000, tuple(pos[k]), ml, delta=tuple(d), beta_inverse=1.0 / rng.uniform(0.75, 0.9999),
                                          time=float(rng.uniform(0.0, 5.0))))
    gs = np.stack(gs)
    N = 120_000
    eng = _engine(fd, phys, max_photon=N, num_sensor=scenes.NUM_PMT)
    res = eng.simulate(gs, 6, sensor_hits=True)
    eng.close()
    assert res["status"] == 0, E.status_names(res["status"])          # LOOP_CAP clear
    assert np.all((res["seq"][:, 0, 0] & 0xF) == 1)                      # CK first
    ph, sq = O.ref_simulate_gpu(fd.arrays(), phys, gs, event_index=6)
    _compare("Cerenkov 120k", res, ph, sq)
