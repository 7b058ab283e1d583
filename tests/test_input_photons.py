"""Input photons (gencode 19, SEvt::setInputPhoton) and carrier gensteps (gencode 14,
scarrier::generate) in the CPU oracle: the generated photon is the given one with the TORCH flag,
and the carrier photon steps 10 mm in y per photon index."""
import numpy as np

from oracle import oracle as O
from opticks_b200 import scenes


def _box():
    fd, lib, _, _ = scenes.sphere_in_box(1)
    return fd.arrays(), lib.arrays()


def test_oracle_input_photons_start_as_given():
    geo, phys = _box()
    n = 64
    inp = scenes.input_photons(n, seed=3)
    S = O.Scene(geo, phys, max_bounce=0, input_photon=inp)
    gs = scenes.input_photon_genstep(n)[None]
    u = np.random.default_rng(0).random((n, 64), dtype=np.float32)
    ph, sq, err = S.simulate(gs, u, 0)
    assert err == 0
    np.testing.assert_array_equal(ph[:, :3, :], inp[:, :3, :])          # max_bounce 0: the start point
    flags = ph.view(np.uint32)[:, 3, 0] & 0xffff
    assert np.all(flags == 0x4) and np.all(ph.view(np.uint32)[:, 3, 3] & 0x4)
    np.testing.assert_array_equal(ph.view(np.uint32)[:, 3, 2], np.arange(n, dtype=np.uint32))   # set_index
    assert np.all((sq[:, 0, 0] & 0xF) == 3)                              # TO first nibble


def test_oracle_input_photons_propagate():
    geo, phys = _box()
    n = 200
    inp = scenes.input_photons(n, seed=4)
    S = O.Scene(geo, phys, input_photon=inp)
    u = np.random.default_rng(1).random((n, 256), dtype=np.float32)
    ph, sq, err = S.simulate(scenes.input_photon_genstep(n)[None], u, 0)
    assert err == 0
    # every photon leaves the water sphere and ends on the detecting box or is absorbed on the way
    assert np.mean((ph.view(np.uint32)[:, 3, 3] & 0x40) != 0) > 0.3


def test_oracle_carrier_steps_in_y():
    geo, phys = _box()
    n = 5
    gs = scenes.carrier_genstep(n, pos=(1.0, 2.0, 3.0), time=0.5, mom=(0.0, 0.0, 1.0), pol=(1.0, 0.0, 0.0), wavelength=450.0)[None]
    S = O.Scene(geo, phys, max_bounce=0)
    ph, sq, err = S.simulate(gs, np.zeros((n, 8), np.float32), 0)
    assert err == 0
    np.testing.assert_allclose(ph[:, 0, 1], 2.0 + 10.0 * np.arange(n))
    np.testing.assert_allclose(ph[:, 1, :3], np.tile([0.0, 0.0, 1.0], (n, 1)))
    assert np.all(ph[:, 2, 3] == 450.0)
    assert np.all((ph.view(np.uint32)[:, 3, 0] & 0xffff) == 0x4)


def test_reference_driver_needs_the_input_photons():
    gs = scenes.input_photon_genstep(10)[None]
    import pytest
    with pytest.raises(ValueError):
        O.ref_genstep_check(gs)
    O.ref_genstep_check(gs, have_input=True)


def test_planck_table_matches_reference_golden():
    # QPlanck's black-body wavelength ICDF: the engine's and the oracle's restatements against the
    # reference's own sblackbody table
    import os
    from tests.conftest import ROOT
    from opticks_b200 import engine as E
    ref = np.load(os.path.join(ROOT, "tests", "golden", "planck_icdf_ref.npy"))
    np.testing.assert_array_equal(O.planck_icdf(), ref)
    np.testing.assert_array_equal(E.planck_icdf(), ref)
    assert ref[0] == 80.0 and np.all(np.diff(ref) >= 0.0) and ref[-1] < 800.0


def test_oracle_torch_without_wavelength_samples_black_body():
    geo, phys = _box()
    n = 400
    gs = scenes.torch_genstep(n, wavelength=0.0, type_=scenes.T_SPHERE)[None]
    S = O.Scene(geo, phys, max_bounce=0)
    u = np.random.default_rng(5).random((n, 16), dtype=np.float32)
    ph, sq, err = S.simulate(gs, u, 0)
    wl = ph[:, 2, 3]
    assert np.all((wl > 80.0) & (wl < 800.0))
    assert 300.0 < np.median(wl) < 700.0          # 6500 K peaks near 446 nm
