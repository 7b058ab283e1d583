"""The engine built from arrays read back from the reference's on-disk layout simulates exactly
as the engine built from the in-memory arrays."""
import numpy as np
import pytest

from opticks_b200 import loader, scenes

pytestmark = pytest.mark.gpu


def test_engine_from_loaded_geometry(cuda, tmp_path):
    from opticks_b200 import engine as E
    fd, lib, icdf = scenes.detector()
    phys = lib.arrays()
    phys["icdf"] = icdf
    loader.save_geom(str(tmp_path), fd.arrays(), phys)
    g2, p2 = loader.load_geom(str(tmp_path))
    gs = scenes.detector_gensteps(4, 2500, seed=8, lib=lib)
    cfg = E.default_config(max_photon=10000, num_sensor=scenes.NUM_PMT)
    a = E.Engine(fd.arrays(), phys, cfg)
    b = E.Engine(g2, p2, cfg)
    ra, rb = a.simulate(gs, 2, sensor_hits=True), b.simulate(gs, 2, sensor_hits=True)
    a.close(); b.close()
    assert ra["num_hit"] > 0 and ra["status"] == 0
    assert np.array_equal(ra["photon"].view(np.uint32), rb["photon"].view(np.uint32))
    assert np.array_equal(ra["seq"], rb["seq"])
    assert np.array_equal(ra["sensor_hits"], rb["sensor_hits"])


def test_engine_from_reference_written_files(cuda):
    """the engine built from tests/golden/npfold (written by the reference's NP.hh) simulates exactly
    as the engine built from the arrays it was made from"""
    import os
    import sys
    from opticks_b200 import engine as E
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.join(here, "golden"))
    from make_npfold import fixture_scene
    geom, phys, _ = fixture_scene()
    g2, p2 = loader.load_geom(os.path.join(here, "golden", "npfold"))
    gs = scenes.torch_genstep(20000, type_=scenes.T_SPHERE, distance=0.25)[None]
    cfg = E.default_config(max_photon=20000)
    a = E.Engine(geom, phys, cfg)
    b = E.Engine(g2, p2, cfg)
    ra, rb = a.simulate(gs, 1), b.simulate(gs, 1)
    a.close(); b.close()
    assert ra["status"] == 0 and ra["num_hit"] > 1000
    assert np.array_equal(ra["photon"].view(np.uint32), rb["photon"].view(np.uint32))
    assert np.array_equal(ra["seq"], rb["seq"])
