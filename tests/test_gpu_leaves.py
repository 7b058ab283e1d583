"""The further CSG leaves on the GPU (cone, hyperboloid, convexpolyhedron with its plan table,
phicut, halfspace): scans against the reference's own device intersector (same device, same
fast-math flags), and a whole simulation through bodies made of them against the reference's
qsim and the CPU oracle."""
import numpy as np
import pytest

from oracle import oracle as O
from opticks_b200 import scenes
from tests._parity import describe, frac_close, seq_match

pytestmark = pytest.mark.gpu

SEQ_BAR = 0.999
TOL = 1e-4


@pytest.fixture(scope="module")
def zoo(cuda):
    from opticks_b200 import engine as E
    fd, prims = scenes.csg_leaf_zoo()
    _, lib, _, _ = scenes.sphere_in_box(1)
    eng = E.Engine(fd.arrays(), lib.arrays(), E.default_config(max_photon=1024))
    yield eng, fd.arrays(), prims
    eng.close()


@pytest.mark.skipif(not O.have_ref_sim(), reason="reference GPU build absent")
def test_further_leaves_match_reference_device_code(zoo):
    eng, A, prims = zoo
    rays = scenes.scan_rays(1 << 17, seed=9, half=400.0)
    for k, p in enumerate(prims):
        if k in scenes.ZOO_EXTRA_PRIMS:
            continue
        root = int(A["prim"].view(np.int32)[p, 0, 1])
        ref = O.ref_scan_gpu(A["node"], A["itra"], root, rays, 0.0, plan=A["plan"])
        out = eng.scan(p, rays, 0.0)
        hr, ho = ref[:, 3] > 0, out[:, 3] > 0
        mism = int((hr != ho).sum())
        exact = float(np.mean(np.all(ref == out, axis=1)))
        both = hr & ho
        rel = np.abs(out[both, 3] - ref[both, 3]) / np.maximum(ref[both, 3], 1.0)
        print(f"zoo prim {k}: hits {hr.sum()} mismatches {mism} bit-exact {exact:.6f} t rel max {rel.max():.3g}")
        assert hr.sum() > 1000, k
        assert mism <= 2, k
        assert np.quantile(rel, 0.999) < 1e-5, k
        assert rel.max() < 1e-3, k


@pytest.fixture(scope="module")
def zoo_sim(cuda):
    from opticks_b200 import engine as E
    n = 200_000
    fd, lib, _, gs = scenes.leaf_zoo_detector(n)      # reference torch type: sphere
    phys = lib.arrays()
    eng = E.Engine(fd.arrays(), phys, E.default_config(max_photon=n))
    res = eng.simulate(gs, 0)
    yield dict(fd=fd, phys=phys, gs=gs, eng=eng, res=res, n=n)
    eng.close()


def test_zoo_simulation_runs_clean(zoo_sim):
    from opticks_b200 import engine as E
    r = zoo_sim["res"]
    assert r["status"] == 0, E.status_names(r["status"])
    assert r["num_hit"] > zoo_sim["n"] // 2
    # most photons cross at least one acrylic body before the walls: more than 2 steps
    nib = np.array([(r["seq"][:, 0, 0] >> (4 * k)) & 0xF for k in range(16)]).T
    assert np.mean((nib != 0).sum(1) > 2) > 0.1


@pytest.mark.skipif(not O.have_ref_sim(), reason="reference GPU build absent")
def test_zoo_simulation_matches_reference_device_code(zoo_sim):
    ph, sq = O.ref_simulate_gpu(zoo_sim["fd"].arrays(), zoo_sim["phys"], zoo_sim["gs"])
    r = zoo_sim["res"]
    m = seq_match(r["seq"], sq)
    same = np.all(r["seq"][:, 0, :] == sq[:, 0, :], axis=1)
    fc = frac_close(r["photon"], ph, same, TOL)
    print(f"leaf zoo vs reference: seqhis match {m:.6f} close {fc:.6f} ({describe(r['photon'], ph, same, TOL)})")
    assert m >= SEQ_BAR
    assert fc >= SEQ_BAR
    np.testing.assert_array_equal(r["seq"][same, 1, :], sq[same, 1, :])


def test_zoo_simulation_matches_cpu_oracle(zoo_sim):
    n = 4000
    u = zoo_sim["eng"].rng_sequence(0, 0, n, 1024)
    S = O.Scene(zoo_sim["fd"].arrays(), zoo_sim["phys"])
    ph, sq, err = S.simulate(zoo_sim["gs"], u, 0)
    assert err & 1 == 0
    r = zoo_sim["res"]
    m = seq_match(r["seq"][:n], sq)
    same = np.all(r["seq"][:n, 0, :] == sq[:, 0, :], axis=1)
    fc = frac_close(r["photon"][:n], ph, same, TOL)
    print(f"leaf zoo vs CPU oracle: seqhis match {m:.6f} close {fc:.6f}")
    assert m >= 0.995
    assert fc >= 0.995


def test_polyhedron_behind_the_ray_is_no_hit(cuda):
    """photons start inside an octahedron's bounding box but outside the solid and move away from
    it: the reference leaf reports valid with t = 0 there, which the trace must drop (OptiX's
    [tmin, tmax] rule), so every photon reaches the detecting wall with a finite direction"""
    from opticks_b200 import engine as E, foundry as F
    import math
    lib = scenes.M.BoundaryLib()
    lib.mat(scenes.VACUUM)
    lib.mat(scenes.M.Material("Rock", rindex=1.5, absorption_length=1.0, scattering_length=1e9))
    lib.mat(scenes.M.Material("Acrylic", rindex=1.49, absorption_length=1e6, scattering_length=1e6))
    lib.sur(scenes.M.Surface("Detector", detect=1.0, absorb=0.0))
    b_box = lib.add("Rock", "", "Detector", "Vacuum")
    b_acr = lib.add("Vacuum", "", "", "Acrylic")
    octa = [(sx / math.sqrt(3.0), sy / math.sqrt(3.0), sz / math.sqrt(3.0), 180.0)
            for sx in (-1, 1) for sy in (-1, 1) for sz in (-1, 1)]
    fd = F.Foundry()
    prims = [fd.add_prim(F.box3(3000.0, 3000.0, 3000.0), b_box),
             fd.add_prim(F.convexpolyhedron(octa, (-312, -312, -312, 312, 312, 312)), b_acr)]
    fd.add_inst(np.eye(4), fd.add_solid("octa", prims))
    n = 1000
    gs = scenes.torch_genstep(n, pos=(250.0, 250.0, 250.0), mom=(1.0, 0.8, 0.6), type_=scenes.T_POINT)[None]
    phys = lib.arrays()
    eng = E.Engine(fd.arrays(), phys, E.default_config(max_photon=n))
    r = eng.simulate(gs, 0)
    eng.close()
    assert r["status"] == 0, E.status_names(r["status"])
    assert np.isfinite(r["photon"][:, 1, :3]).all()
    assert r["num_hit"] == n
    S = O.Scene(fd.arrays(), phys)
    u = np.random.default_rng(3).random((n, 256), dtype=np.float32)
    ph, sq, err = S.simulate(gs, u, 0)
    assert err & 1 == 0 and np.isfinite(ph[:, 1, :3]).all()
    if O.have_ref_sim():
        ph, sq = O.ref_simulate_gpu(fd.arrays(), phys, gs)
        assert np.isfinite(ph[:, 1, :3]).all()
        np.testing.assert_array_equal(sq[:, 0, :], r["seq"][:, 0, :])
