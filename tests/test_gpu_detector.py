"""Full synthetic detector (17,612 instanced PMTs, scintillation with reemission) on the GPU:
the BVH traversal + CSG + physics against the reference's device code (brute-force closest hit
over all instances) and the CPU oracle, plus per-sensor hit counts."""
import numpy as np
import pytest

from oracle import oracle as O
from opticks_b200 import scenes
from tests._parity import frac_close, seq_match

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def det(cuda):
    from opticks_b200 import engine as E
    fd, lib, icdf = scenes.detector()
    phys = lib.arrays()
    phys["icdf"] = icdf
    gs = scenes.detector_gensteps(2, 1000, seed=1, lib=lib)
    eng = E.Engine(fd.arrays(), phys, E.default_config(max_photon=2000, num_sensor=scenes.NUM_PMT))
    res = eng.simulate(gs, 0, sensor_hits=True)
    yield dict(fd=fd, lib=lib, phys=phys, gs=gs, eng=eng, res=res)
    eng.close()


def test_detector_runs_clean(det):
    from opticks_b200 import engine as E
    r = det["res"]
    assert r["status"] == 0, E.status_names(r["status"])
    assert r["num_hit"] > 100
    sh = r["sensor_hits"]
    assert sh.sum() == r["num_hit"]
    ids = r["hit"].view(np.uint32)[:, 3, 1] & 0xFFFFFF
    np.testing.assert_array_equal(np.bincount(ids - 1, minlength=scenes.NUM_PMT), sh)


@pytest.mark.skipif(not O.have_ref_sim(), reason="reference GPU build absent")
def test_detector_matches_reference_device_code(det):
    ph, sq = O.ref_simulate_gpu(det["fd"].arrays(), det["phys"], det["gs"])
    r = det["res"]
    m = seq_match(r["seq"], sq)
    same = np.all(r["seq"][:, 0, :] == sq[:, 0, :], axis=1)
    fc = frac_close(r["photon"], ph, same, 1e-4)
    print(f"detector vs reference: seqhis match {m:.6f} close {fc:.6f}")
    assert m >= 0.999
    assert fc >= 0.999


def test_detector_matches_cpu_oracle(det):
    n = 600
    u = det["eng"].rng_sequence(0, 0, n, 1024)
    S = O.Scene(det["fd"].arrays(), det["phys"])
    ph, sq, err = S.simulate(det["gs"], u, 0)
    assert err & 1 == 0
    r = det["res"]
    m = seq_match(r["seq"][:n], sq)
    same = np.all(r["seq"][:n, 0, :] == sq[:, 0, :], axis=1)
    fc = frac_close(r["photon"][:n], ph, same, 1e-4)
    print(f"detector vs CPU oracle: seqhis match {m:.6f} close {fc:.6f}")
    assert m >= 0.995
    assert fc >= 0.995


@pytest.fixture(scope="module")
def ck(cuda):
    """Cerenkov gensteps (tracks of beta 0.99, 0.8, 0.999 in the liquid scintillator): the
    bnd-texture rejection sampling of wavelength and cone angle, and the fraction/delta sampling
    along the step"""
    from opticks_b200 import engine as E
    fd, lib, icdf = scenes.detector()
    phys = lib.arrays()
    phys["icdf"] = icdf
    ml = lib.material_line("LS")
    rng = np.random.default_rng(17)
    gs = np.stack([scenes.cerenkov_genstep(700, tuple(scenes.uniform_ball(1, 15000.0, rng)[0]), ml,
                                           delta=tuple(rng.normal(size=3) * 4.0), beta_inverse=b, time=1.5 * k)
                   for k, b in enumerate((1.0 / 0.99, 1.0 / 0.8, 1.0 / 0.999))])
    eng = E.Engine(fd.arrays(), phys, E.default_config(max_photon=4096, num_sensor=scenes.NUM_PMT))
    res = eng.simulate(gs, 0, sensor_hits=True)
    yield dict(fd=fd, phys=phys, gs=gs, eng=eng, res=res)
    eng.close()


def test_cerenkov_generation(ck):
    from opticks_b200 import engine as E
    r = ck["res"]
    assert r["status"] == 0, E.status_names(r["status"])
    assert np.all((r["seq"][:, 0, 0] & 0xF) == 1)              # CK is the first history nibble
    wl = r["photon"][:, 2, 3]
    assert np.all((wl >= 300.0 - 1e-3) & (wl <= 600.0 + 1e-3))


@pytest.mark.skipif(not O.have_ref_sim(), reason="reference GPU build absent")
def test_cerenkov_matches_reference_device_code(ck):
    ph, sq = O.ref_simulate_gpu(ck["fd"].arrays(), ck["phys"], ck["gs"])
    r = ck["res"]
    m = seq_match(r["seq"], sq)
    same = np.all(r["seq"][:, 0, :] == sq[:, 0, :], axis=1)
    fc = frac_close(r["photon"], ph, same, 1e-4)
    print(f"cerenkov vs reference: seqhis match {m:.6f} close {fc:.6f}")
    assert m >= 0.999
    assert fc >= 0.999


def test_cerenkov_matches_cpu_oracle(ck):
    n = 800
    u = ck["eng"].rng_sequence(0, 0, n, 1024)
    S = O.Scene(ck["fd"].arrays(), ck["phys"])
    ph, sq, err = S.simulate(ck["gs"], u, 0)
    assert err & 1 == 0
    r = ck["res"]
    m = seq_match(r["seq"][:n], sq)
    same = np.all(r["seq"][:n, 0, :] == sq[:, 0, :], axis=1)
    fc = frac_close(r["photon"][:n], ph, same, 1e-4)
    print(f"cerenkov vs CPU oracle: seqhis match {m:.6f} close {fc:.6f}")
    assert m >= 0.995
    assert fc >= 0.995


@pytest.mark.parametrize("mode", [1, 2])
def test_pinned_outputs_equal_pageable(det, mode):
    """phx_simulate writes photons and seq straight into pinned (device-mapped) host buffers while
    the kernels run; the result equals the staged copy into pageable buffers"""
    import torch
    from opticks_b200 import engine as E
    gs = det["gs"]
    N = int(gs.view(np.int32)[:, 0, 3].sum())
    eng = E.Engine(det["fd"].arrays(), det["phys"], E.default_config(max_photon=N, num_sensor=scenes.NUM_PMT, kernel_mode=mode))
    ref = eng.simulate(gs, 4, sensor_hits=True)
    ph = torch.empty((N, 4, 4), dtype=torch.float32, pin_memory=True).numpy()
    sq = torch.empty((N, 2, 2), dtype=torch.int64, pin_memory=True).numpy().view(np.uint64)
    ht = torch.empty((N, 4, 4), dtype=torch.float32, pin_memory=True).numpy()
    ph.fill(7.0)
    out = eng.simulate_into(gs, 4, ph, sq, ht)
    eng.close()
    assert out["status"] == 0 and out["num_hit"] == ref["num_hit"]
    np.testing.assert_array_equal(ph.view(np.uint32), ref["photon"].view(np.uint32))
    np.testing.assert_array_equal(sq, ref["seq"])
    np.testing.assert_array_equal(ht[: out["num_hit"]].view(np.uint32), ref["hit"].view(np.uint32))
