"""CSG scan on the GPU (CSGScan): the CUDA intersector against the reference's own intersector
(same device, same fast-math flags), the committed golden vectors, and the FP64 oracle."""
import os

import numpy as np
import pytest

from tests.conftest import ROOT
from oracle import oracle as O
from opticks_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tree_engine(cuda):
    from opticks_b200 import engine as E
    fd, p = scenes.csg_scan_tree(with_torus=True)
    _, lib, _, _ = scenes.sphere_in_box(1)
    eng = E.Engine(fd.arrays(), lib.arrays(), E.default_config(max_photon=1024))
    yield eng, fd.arrays(), p
    eng.close()


@pytest.fixture(scope="module")
def notorus_engine(cuda):
    from opticks_b200 import engine as E
    fd, p = scenes.csg_scan_tree(with_torus=False)
    _, lib, _, _ = scenes.sphere_in_box(1)
    eng = E.Engine(fd.arrays(), lib.arrays(), E.default_config(max_photon=1024))
    yield eng, fd.arrays(), p
    eng.close()


def test_scan_golden_reference_vectors(cuda):
    from opticks_b200 import engine as E
    g = np.load(os.path.join(ROOT, "tests", "golden", "csg_scan_ref.npz"))
    # rebuild a foundry around the golden node table (one prim per root)
    _, lib, _, _ = scenes.sphere_in_box(1)
    for key, roots, rays, ref in (("tree", [int(g["tree_root"])], g["tree_rays"], g["tree_isect"][None]),
                                  ("leaf", list(g["leaf_roots"]), g["leaf_rays"], g["leaf_isect"])):
        node = g[f"{key}_node"]
        prim = np.zeros((len(roots), 4, 4), np.float32)
        pi = prim.view(np.int32)
        for k, r in enumerate(roots):
            nn = node.view(np.uint32)[r, 0, 0] if node.view(np.uint32)[r, 3, 2] < 11 else 1
            pi[k, 0, 0] = max(1, nn)
            pi[k, 0, 1] = r
            prim[k, 2, :] = (-1000, -1000, -1000, 1000)
            prim[k, 3, :2] = (1000, 1000)
        solid = np.zeros((1, 3, 4), np.int32)
        solid[0, 1, 0] = len(roots)
        inst = np.eye(4, dtype=np.float32)[None].copy()
        geo = dict(node=node, prim=prim, solid=solid, inst=inst, itra=g[f"{key}_itra"])
        eng = E.Engine(geo, lib.arrays(), E.default_config(max_photon=64))
        for k in range(len(roots)):
            out = eng.scan(k, rays, 0.0)
            hr, ho = ref[k][:, 3] > 0, out[:, 3] > 0
            assert (hr != ho).sum() == 0, (key, k)
            np.testing.assert_allclose(out[hr, 3], ref[k][hr, 3], rtol=1e-4, atol=1e-4)
            np.testing.assert_allclose(out[hr, :3], ref[k][hr, :3], atol=1e-5)
        eng.close()


@pytest.mark.skipif(not O.have_ref_sim(), reason="reference GPU build absent")
def test_scan_matches_reference_device_code(notorus_engine):
    eng, A, p = notorus_engine
    root = int(A["prim"].view(np.int32)[p, 0, 1])
    rays = scenes.scan_rays(1 << 18, seed=1, half=600.0)
    ref = O.ref_scan_gpu(A["node"], A["itra"], root, rays, 0.0)
    out = eng.scan(p, rays, 0.0)
    hr, ho = ref[:, 3] > 0, out[:, 3] > 0
    mism = int((hr != ho).sum())
    exact = float(np.mean(np.all(ref == out, axis=1)))
    print(f"scan vs reference device code: hits {hr.sum()} hit/miss mismatches {mism} bit-exact {exact:.6f}")
    assert mism <= 2
    both = hr & ho
    rel = np.abs(out[both, 3] - ref[both, 3]) / np.maximum(ref[both, 3], 1.0)
    # grazing rays make the quadratic root ill-conditioned: one ulp of the discriminant moves t
    print(f"   t rel diff p99.9 {np.quantile(rel, 0.999):.3g} max {rel.max():.3g}")
    assert np.quantile(rel, 0.999) < 1e-5
    assert rel.max() < 1e-3
    assert exact > 0.95


def test_scan_with_torus_against_fp64_oracle(tree_engine):
    eng, A, p = tree_engine
    root = int(A["prim"].view(np.int32)[p, 0, 1])
    rays = scenes.scan_rays(1 << 17, seed=2, half=500.0)
    out = eng.scan(p, rays, 0.0)
    t64, err = O.csg_scan_t64(A["node"], A["itra"], root, rays, 0.0)
    assert err == 0
    hg, h64 = out[:, 3] > 0, t64 > 0
    mism = int((hg != h64).sum())
    both = hg & h64
    rel = np.abs(out[both, 3] - t64[both]) / np.maximum(t64[both], 1.0)
    print(f"torus tree: hits {both.sum()} mismatches {mism} rel err max {rel.max():.3g} p99.9 {np.quantile(rel, 0.999):.3g}")
    assert both.sum() > 1000
    assert mism <= max(3, int(2e-4 * len(rays)))
    assert np.quantile(rel, 0.999) < 1e-4


def test_scan_polish_reduces_distance_error(tree_engine, cuda):
    import torch
    eng, A, p = tree_engine
    root = int(A["prim"].view(np.int32)[p, 0, 1])
    rays = scenes.scan_rays(1 << 16, seed=4, half=800.0)
    t64, _ = O.csg_scan_t64(A["node"], A["itra"], root, rays, 0.0)
    r = torch.from_numpy(rays).cuda()
    res = {}
    for pol in (0, 1):
        o = torch.zeros((rays.shape[1], 4), device="cuda")
        eng.scan_device(p, r, rays.shape[1], o, 0.0, pol)
        torch.cuda.synchronize()
        o = o.cpu().numpy()
        both = (o[:, 3] > 0) & (t64 > 0)
        res[pol] = np.abs(o[both, 3] - t64[both]).max()
    print("max |t - t64| without/with FP64 polish", res)
    assert res[1] <= res[0] + 1e-6


def test_scan_edge_cases(notorus_engine):
    eng, A, p = notorus_engine
    # empty scan, axis-aligned rays, rays starting on a surface
    assert eng.scan(p, np.zeros((6, 0), np.float32)).shape == (0, 4)
    o = np.array([[0, 0, 1000], [1000, 0, 0], [0, 0, 0], [0, 0, 190]], np.float32)
    d = np.array([[0, 0, -1], [-1, 0, 0], [0, 0, 1], [0, 0, 1]], np.float32)
    rays = np.ascontiguousarray(np.concatenate([o.T, d.T]))
    out = eng.scan(p, rays, 0.0)
    t, _ = O.csg_scan(A["node"], A["itra"], int(A["prim"].view(np.int32)[p, 0, 1]), rays, 0.0)
    np.testing.assert_array_equal(out[:, 3] > 0, t[:, 3] > 0)
    np.testing.assert_allclose(out[:, 3], t[:, 3], rtol=1e-6)


@pytest.fixture(scope="module")
def zoo_engine(cuda):
    from opticks_b200 import engine as E
    fd, prims = scenes.csg_leaf_zoo()
    _, lib, _, _ = scenes.sphere_in_box(1)
    eng = E.Engine(fd.arrays(), lib.arrays(), E.default_config(max_photon=1024))
    yield eng, fd.arrays(), prims
    eng.close()


def test_scan_further_leaves_match_reference_golden(zoo_engine):
    """cone, hyperboloid, convexpolyhedron (plan table), phicut, halfspace trees against the
    intersects of the reference's own tree intersector"""
    eng, A, prims = zoo_engine
    g = np.load(os.path.join(ROOT, "tests", "golden", "csg_zoo_ref.npz"))
    np.testing.assert_array_equal(A["node"], g["node"])
    for k, p in enumerate(g["prims"]):
        ref = g["isect"][k]
        out = eng.scan(int(p), g["rays"], 0.0)
        hr, ho = ref[:, 3] > 0, out[:, 3] > 0
        mism = int((hr != ho).sum())
        assert mism <= 2, (int(p), mism)
        both = hr & ho
        np.testing.assert_allclose(out[both, 3], ref[both, 3], rtol=1e-4, atol=1e-4, err_msg=f"prim {int(p)}")
        np.testing.assert_allclose(out[both, :3], ref[both, :3], atol=2e-5, err_msg=f"prim {int(p)}")


def test_scan_extra_leaf_trees_match_oracle(zoo_engine):
    """trees holding slab / infcylinder / disc leaves against the oracle (pinned leaf by leaf to
    the reference's leaf functions)"""
    eng, A, prims = zoo_engine
    rays = scenes.scan_rays(1 << 15, seed=21, half=400.0)
    for k in scenes.ZOO_EXTRA_PRIMS:
        p = prims[k]
        root = int(A["prim"].view(np.int32)[p, 0, 1])
        ref, err = O.csg_scan(A["node"], A["itra"], root, rays, 0.0, plan=A["plan"])
        assert err == 0
        out = eng.scan(p, rays, 0.0)
        hr, ho = ref[:, 3] > 0, out[:, 3] > 0
        assert hr.sum() > 500, k
        assert int((hr != ho).sum()) <= 3, k
        both = hr & ho
        np.testing.assert_allclose(out[both, 3], ref[both, 3], rtol=1e-4, atol=1e-4, err_msg=f"zoo prim {k}")
        np.testing.assert_allclose(out[both, :3], ref[both, :3], atol=2e-5, err_msg=f"zoo prim {k}")
