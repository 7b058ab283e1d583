"""phx_trim releases the memory an engine grew for its calls (the wavefront path pool above all), and
the next call allocates again and gives the same photons, seq and hits."""
import numpy as np
import pytest

from opticks_b200 import scenes

pytestmark = pytest.mark.gpu


def test_trim_releases_pool_and_next_call_is_identical(cuda):
    import torch
    from opticks_b200 import engine as E
    fd, lib, icdf = scenes.detector()
    phys = lib.arrays()
    phys["icdf"] = icdf
    gs = scenes.detector_gensteps(40, 5000, seed=3, lib=lib)
    N = int(gs.view(np.int32)[:, 0, 3].sum())
    eng = E.Engine(fd.arrays(), phys, E.default_config(max_photon=N, num_sensor=scenes.NUM_PMT))
    a = eng.simulate(gs, 5, sensor_hits=True)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    freed = eng.trim()
    free1 = torch.cuda.mem_get_info()[0]
    assert freed >= N * 180                          # at least one path slot per photon of the call
    assert free1 - free0 >= freed // 2               # the driver sees the memory come back
    assert eng.trim() == 0                           # nothing left to release
    b = eng.simulate(gs, 5, sensor_hits=True)
    eng.close()
    np.testing.assert_array_equal(a["photon"].view(np.uint32), b["photon"].view(np.uint32))
    np.testing.assert_array_equal(a["seq"], b["seq"])
    np.testing.assert_array_equal(a["hit"].view(np.uint32), b["hit"].view(np.uint32))
    np.testing.assert_array_equal(a["sensor_hits"], b["sensor_hits"])
