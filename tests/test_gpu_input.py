"""Input photons (gencode 19) and carrier gensteps (gencode 14) on the GPU against the reference's
own qsim (same device, same cuRAND streams) and the CPU oracle, with the host and device forms of
phx_set_input_photon and the out-of-range status."""
import numpy as np
import pytest

from oracle import oracle as O
from opticks_b200 import scenes
from tests._parity import frac_close, seq_match

pytestmark = pytest.mark.gpu

SEQ_BAR = 0.999
TOL = 1e-4


@pytest.fixture(scope="module")
def box(cuda):
    from opticks_b200 import engine as E
    fd, lib, _, _ = scenes.sphere_in_box(1)
    n = 50_000
    inp = scenes.input_photons(n, seed=11, radius=300.0)
    eng = E.Engine(fd.arrays(), lib.arrays(), E.default_config(max_photon=n))
    eng.set_input_photon(inp)
    gs = scenes.input_photon_genstep(n)[None]
    res = eng.simulate(gs, 0)
    yield dict(fd=fd, phys=lib.arrays(), eng=eng, inp=inp, gs=gs, res=res, n=n)
    eng.close()


def test_input_photons_run_clean(box):
    from opticks_b200 import engine as E
    r = box["res"]
    assert r["status"] == 0, E.status_names(r["status"])
    assert np.all((r["seq"][:, 0, 0] & 0xF) == 3)                     # TO first
    np.testing.assert_array_equal(r["photon"].view(np.uint32)[:, 3, 2], np.arange(box["n"], dtype=np.uint32))


@pytest.mark.skipif(not O.have_ref_sim(), reason="reference GPU build absent")
def test_input_photons_match_reference_device_code(box):
    ph, sq = O.ref_simulate_gpu(box["fd"].arrays(), box["phys"], box["gs"], input_photon=box["inp"])
    r = box["res"]
    m = seq_match(r["seq"], sq)
    same = np.all(r["seq"][:, 0, :] == sq[:, 0, :], axis=1)
    fc = frac_close(r["photon"], ph, same, TOL)
    print(f"input photons vs reference: seqhis match {m:.6f} close {fc:.6f}")
    assert m >= SEQ_BAR
    assert fc >= SEQ_BAR


def test_input_photons_match_cpu_oracle(box):
    n = 2000
    u = box["eng"].rng_sequence(0, 0, n, 1024)
    S = O.Scene(box["fd"].arrays(), box["phys"], input_photon=box["inp"])
    ph, sq, err = S.simulate(scenes.input_photon_genstep(box["n"])[None], u, 0)
    assert err & 1 == 0
    r = box["res"]
    m = seq_match(r["seq"][:n], sq)
    same = np.all(r["seq"][:n, 0, :] == sq[:, 0, :], axis=1)
    assert m >= 0.995
    assert frac_close(r["photon"][:n], ph, same, TOL) >= 0.995


def test_input_photons_from_device_buffer_and_range(box, cuda):
    from opticks_b200 import engine as E
    torch = cuda
    eng = box["eng"]
    dev = torch.from_numpy(box["inp"]).cuda()
    eng.set_input_photon(dev)
    r = eng.simulate(box["gs"], 0)
    np.testing.assert_array_equal(r["seq"], box["res"]["seq"])
    np.testing.assert_array_equal(r["photon"], box["res"]["photon"])
    # more photons asked than given: the rest stay zero and the status says so
    eng.set_input_photon(box["inp"][:100])
    r2 = eng.simulate(scenes.input_photon_genstep(200)[None], 0)
    assert "INPUT_RANGE" in E.status_names(r2["status"])
    eng.set_input_photon(box["inp"])


@pytest.mark.skipif(not O.have_ref_sim(), reason="reference GPU build absent")
def test_carrier_genstep_matches_reference(cuda):
    from opticks_b200 import engine as E
    fd, lib, _, _ = scenes.sphere_in_box(1)
    n = 40
    gs = scenes.carrier_genstep(n, pos=(0.0, -200.0, 0.0), time=0.1, mom=(0.6, 0.0, 0.8), pol=(0.8, 0.0, -0.6), wavelength=450.0)[None]
    eng = E.Engine(fd.arrays(), lib.arrays(), E.default_config(max_photon=n))
    r = eng.simulate(gs, 0)
    eng.close()
    assert r["status"] == 0
    ph, sq = O.ref_simulate_gpu(fd.arrays(), lib.arrays(), gs)
    assert seq_match(r["seq"], sq) >= 0.95
    same = np.all(r["seq"][:, 0, :] == sq[:, 0, :], axis=1)
    assert frac_close(r["photon"], ph, same, TOL) >= 0.95


@pytest.mark.skipif(not O.have_ref_sim(), reason="reference GPU build absent")
def test_torch_without_wavelength_matches_reference(cuda):
    """torch photons without a wavelength take one from the black-body texture (qsim.h:2541-2544)"""
    from opticks_b200 import engine as E
    fd, lib, _, _ = scenes.sphere_in_box(1)
    n = 50_000
    gs = scenes.torch_genstep(n, wavelength=0.0, type_=scenes.T_SPHERE, distance=0.25)[None]
    eng = E.Engine(fd.arrays(), lib.arrays(), E.default_config(max_photon=n))
    r = eng.simulate(gs, 0)
    eng.close()
    assert r["status"] == 0
    wl = r["photon"][:, 2, 3]
    assert np.all((wl > 80.0) & (wl < 800.0))
    ph, sq = O.ref_simulate_gpu(fd.arrays(), lib.arrays(), gs)
    m = seq_match(r["seq"], sq)
    same = np.all(r["seq"][:, 0, :] == sq[:, 0, :], axis=1)
    fc = frac_close(r["photon"], ph, same, TOL)
    wl_exact = float(np.mean(r["photon"][:, 2, 3] == ph[:, 2, 3]))
    print(f"black-body torch vs reference: seqhis {m:.6f} close {fc:.6f} wavelength bit-exact {wl_exact:.6f}")
    assert m >= SEQ_BAR
    assert fc >= SEQ_BAR
