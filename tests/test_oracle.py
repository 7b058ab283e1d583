"""The oracle (oracle/) pinned against the reference: golden intersects produced by the
reference's own CSG intersector, the Kensler decision table, texture-filter emulation and
physics invariants of the CPU restatement."""
import os

import numpy as np
import pytest

from tests.conftest import ROOT
from oracle import oracle as O
from opticks_b200 import engine_module, foundry as F, scenes

GOLD = os.path.join(ROOT, "tests", "golden", "csg_scan_ref.npz")


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


def test_oracle_csg_tree_matches_reference_golden_bit_exact(gold):
    out, err = O.csg_scan(gold["tree_node"], gold["tree_itra"], int(gold["tree_root"]), gold["tree_rays"], 0.0)
    ref = gold["tree_isect"]
    assert err == 0
    assert (ref[:, 3] > 0).sum() > 200
    np.testing.assert_array_equal(out, ref)


def test_oracle_csg_leaves_match_reference_golden_bit_exact(gold):
    for k, root in enumerate(gold["leaf_roots"]):
        out, err = O.csg_scan(gold["leaf_node"], gold["leaf_itra"], int(root), gold["leaf_rays"], 0.0)
        ref = gold["leaf_isect"][k]
        assert err == 0
        assert (ref[:, 3] > 0).sum() > 20, k
        np.testing.assert_array_equal(out, ref, err_msg=f"leaf prim {k}")


@pytest.mark.skipif(not O.have_ref_csg(), reason="reference CPU build absent")
def test_oracle_matches_live_reference_on_fresh_rays():
    fd, p = scenes.csg_scan_tree(with_torus=False)
    A = fd.arrays()
    root = int(A["prim"].view(np.int32)[p, 0, 1])
    rays = scenes.scan_rays(100000, seed=3, half=600.0)
    ref = O.ref_csg_scan(A["node"], A["itra"], root, rays, 0.0)
    out, err = O.csg_scan(A["node"], A["itra"], root, rays, 0.0)
    np.testing.assert_array_equal(out, ref)


def test_kensler_table_rules():
    # spot checks of the single-hit CSG rules (A closer / B closer)
    E, X, M = 0, 1, 2
    act = O.lib().oracle_csg_action
    assert act(1, E, E, 1) == 1 and act(1, E, E, 0) == 2        # union enter/enter : closer
    assert act(1, E, X, 1) == 4 and act(1, X, E, 0) == 5        # union loops
    assert act(1, M, M, 1) == 0
    assert act(2, E, M, 1) == 0 and act(2, X, X, 0) == 2        # intersection
    assert act(3, X, E, 0) == 3 and act(3, E, M, 0) == 1        # difference flips B
    # the packed words of the reference's table (decoded from its published layout)
    words = {(1, 1): 0x22121141, (1, 0): 0x22115122, (2, 1): 0x00014014, (2, 0): 0x00022055,
             (3, 1): 0x00141141, (3, 0): 0x00133155}
    for (op, ac), w in words.items():
        for off in range(8):
            assert act(op, off // 3, off % 3, ac) == (w >> (4 * off)) & 0xF


def test_torus_fp64_hits_analytic_points():
    fd = F.Foundry()
    p = fd.add_prim(F.torus(200.0, 20.0), 0)
    fd.add_solid("t", [p])
    A = fd.arrays()
    # rays along x through the tube centre line at z=0: entry at x = -(R+r) from the far side
    o = np.array([[-1000.0, 0.0, 0.0], [0.0, 0.0, 500.0], [200.0, 0.0, 500.0]], np.float32).T
    d = np.array([[1.0, 0.0, 0.0], [0.0, 0.0, -1.0], [0.0, 0.0, -1.0]], np.float32).T
    rays = np.ascontiguousarray(np.concatenate([o, d]))
    out, err = O.csg_scan(A["node"], A["itra"], 0, rays, 0.0, use_double=True)
    assert err == 0
    assert abs(out[0, 3] - (1000.0 - 220.0)) < 1e-3       # outer equator
    assert out[1, 3] == 0.0                               # down the hole: miss
    assert abs(out[2, 3] - (500.0 - 20.0)) < 1e-3         # top of the tube
    np.testing.assert_allclose(out[2, :3], [0, 0, 1], atol=1e-6)


def test_texture_emulation_linear_and_wrap():
    data = np.arange(8, dtype=np.float32).reshape(1, 8)
    # texel centres reproduce the samples
    for i in range(8):
        assert O.tex2d_f1(data, (i + 0.5) / 8, 0.5) == float(i)
    # halfway between texels 2 and 3
    assert O.tex2d_f1(data, 3.0 / 8, 0.5) == 2.5
    # wrap: below texel 0 blends with the last texel
    assert O.tex2d_f1(data, 0.0, 0.5) == 3.5


def _c1_oracle(n=4000, seed=5, K=256):
    fd, lib, icdf, gs = scenes.sphere_in_box(n)
    S = O.Scene(fd.arrays(), lib.arrays())
    u = np.random.default_rng(seed).random((n, K), dtype=np.float32)
    return S.simulate(gs, u)


def test_oracle_physics_invariants_sphere_in_box():
    ph, seq, err = _c1_oracle()
    assert err == 0
    mom, pol = ph[:, 1, :3], ph[:, 2, :3]
    np.testing.assert_allclose(np.linalg.norm(mom, axis=1), 1.0, atol=2e-5)
    np.testing.assert_allclose(np.linalg.norm(pol, axis=1), 1.0, atol=2e-5)
    assert np.abs((mom * pol).sum(1)).max() < 2e-4
    flags = ph.view(np.uint32)[:, 3, 3]
    E = engine_module()
    lab = [E.seqhis_label(int(s[0, 0]), int(s[0, 1])) for s in seq]
    sd = (flags & 0x40) != 0
    # every detected photon ends on the box wall (|coordinate| = 1500 mm on one axis)
    assert np.allclose(np.abs(ph[sd, 0, :3]).max(1), 1500.0, atol=0.05)
    assert all(l.endswith("SD") for l, s in zip(lab, sd) if s)
    assert all(l.startswith("TO") for l in lab)
    # bulk absorption in 1 m of water with a 10 m absorption length: ~9.5 %
    ab = np.mean([l.endswith("AB") for l in lab])
    assert 0.06 < ab < 0.14
    # seqhis nibbles are consistent with the flagmask
    for s, fm in zip(seq[:500], flags[:500]):
        nib = [(int(s[0, 0]) >> (4 * k)) & 0xF for k in range(16)]
        m = 0
        for v in nib:
            if v:
                m |= 1 << (v - 1)
        assert m == fm


def test_oracle_reports_exhausted_uniform_stream():
    ph, seq, err = _c1_oracle(n=200, K=3)
    assert err & 2


ZOO = os.path.join(ROOT, "tests", "golden", "csg_zoo_ref.npz")


def one_leaf_node(q8, typecode):
    """a one-node table holding leaf (q0, q1) with the given typecode, untransformed"""
    node = np.zeros((1, 4, 4), np.float32)
    node[0, :2] = np.asarray(q8, np.float32).reshape(2, 4)
    node.view(np.uint32)[0, 3, 2] = typecode
    return node


def test_oracle_further_leaves_match_reference_golden_bit_exact():
    g = np.load(ZOO)
    fd, prims = scenes.csg_leaf_zoo()
    A = fd.arrays()
    np.testing.assert_array_equal(A["node"], g["node"])     # the fixture's geometry is the zoo's
    np.testing.assert_array_equal(A["plan"], g["plan"])
    for k, root in enumerate(g["roots"]):
        out, err = O.csg_scan(g["node"], g["itra"], int(root), g["rays"], 0.0, plan=g["plan"])
        ref = g["isect"][k]
        assert err == 0
        assert (ref[:, 3] > 0).sum() > 50, k
        np.testing.assert_array_equal(out, ref, err_msg=f"zoo prim {int(g['prims'][k])}")


def test_oracle_extra_leaves_match_reference_leaf_functions_bit_exact():
    g = np.load(ZOO)
    for k, tc in enumerate(g["extra_typecode"]):
        out, err = O.csg_scan(one_leaf_node(g["extra_q"][k], int(tc)), None, 0, g["rays"], 0.0)
        ref = g["extra_isect"][k]
        assert err == 0
        assert (ref[:, 3] > 0).sum() > 50, k
        np.testing.assert_array_equal(out, ref, err_msg=f"typecode {int(tc)}")


@pytest.mark.skipif(not O.have_ref_csg(), reason="reference CPU build absent")
def test_oracle_further_leaves_match_live_reference_on_fresh_rays():
    fd, prims = scenes.csg_leaf_zoo()
    A = fd.arrays()
    rays = scenes.scan_rays(20000, seed=5, half=400.0)
    for k, p in enumerate(prims):
        if k in scenes.ZOO_EXTRA_PRIMS:
            continue
        root = int(A["prim"].view(np.int32)[p, 0, 1])
        ref = O.ref_csg_scan(A["node"], A["itra"], root, rays, 0.0, plan=A["plan"])
        out, err = O.csg_scan(A["node"], A["itra"], root, rays, 0.0, plan=A["plan"])
        assert err == 0
        np.testing.assert_array_equal(out, ref, err_msg=f"zoo prim {k}")


def test_convexpolyhedron_cube_equals_box():
    # a convexpolyhedron of the six cube planes is the box leaf of the same size
    cube = F.Foundry()
    p0 = cube.add_prim(F.convexpolyhedron(F.cube_planes(150.0), (-150, -150, -150, 150, 150, 150)), 0)
    p1 = cube.add_prim(F.box3(300.0, 300.0, 300.0), 0)
    A = cube.arrays()
    rays = scenes.scan_rays(5000, seed=17, half=400.0)
    r0, r1 = (int(A["prim"].view(np.int32)[p, 0, 1]) for p in (p0, p1))
    a, _ = O.csg_scan(A["node"], A["itra"], r0, rays, 0.0, plan=A["plan"])
    b, _ = O.csg_scan(A["node"], A["itra"], r1, rays, 0.0, plan=A["plan"])
    assert ((a[:, 3] > 0) != (b[:, 3] > 0)).sum() == 0
    np.testing.assert_allclose(a[:, 3], b[:, 3], rtol=1e-5, atol=1e-3)


def test_reference_driver_refuses_gensteps_it_cannot_generate():
    # checked on the host before any launch: an engine-only torch type and an unknown gencode are
    # refused; reference torch types pass, also without a wavelength (the driver sets up QPlanck)
    ok = scenes.torch_genstep(10, type_=scenes.T_SPHERE)[None]
    O.ref_genstep_check(ok)
    with pytest.raises(ValueError):
        O.ref_genstep_check(scenes.torch_genstep(10, type_=scenes.T_SPHERE_RANDPOL)[None])
    O.ref_genstep_check(scenes.torch_genstep(10, wavelength=0.0, type_=scenes.T_SPHERE)[None])   # black-body
    odd = ok.copy()
    odd.view(np.int32)[0, 0, 0] = 99
    with pytest.raises(ValueError):
        O.ref_genstep_check(odd)


LISTS = os.path.join(ROOT, "tests", "golden", "csg_list_ref.npz")


def test_oracle_list_nodes_match_reference_golden_bit_exact():
    g = np.load(LISTS)
    fd, prims = scenes.csg_list_zoo()
    A = fd.arrays()
    np.testing.assert_array_equal(A["node"], g["node"])
    for k, root in enumerate(g["roots"]):
        out, err = O.csg_scan(g["node"], g["itra"], int(root), g["rays"], 0.0, plan=g["plan"])
        ref = g["isect"][k]
        assert err == 0
        assert (ref[:, 3] > 0).sum() > 30, k
        np.testing.assert_array_equal(out, ref, err_msg=f"list prim {k}")


@pytest.mark.skipif(not O.have_ref_csg(), reason="reference CPU build absent")
def test_oracle_list_nodes_match_live_reference_on_fresh_rays():
    fd, prims = scenes.csg_list_zoo()
    A = fd.arrays()
    rays = scenes.scan_rays(20000, seed=23, half=400.0)
    for k, p in enumerate(prims):
        root = int(A["prim"].view(np.int32)[p, 0, 1])
        ref = O.ref_csg_scan(A["node"], A["itra"], root, rays, 0.0, plan=A["plan"])
        out, err = O.csg_scan(A["node"], A["itra"], root, rays, 0.0, plan=A["plan"])
        np.testing.assert_array_equal(out, ref, err_msg=f"list prim {k}")


def test_list_layout_follows_the_reference():
    # a list at the root: header (subNum, subOffset 1) then its leaves; inside a tree the leaves
    # follow the complete binary tree and subOffset counts from the tree's root
    fd = F.Foundry()
    l1 = F.list_node("discontiguous", [F.sphere(10.0), F.translate(F.sphere(10.0), 30.0, 0.0, 0.0)])
    p0 = fd.add_prim(l1, 0)
    p1 = fd.add_prim(F.op("union", F.box3(50.0, 50.0, 50.0), F.list_node("overlap", [F.sphere(20.0), F.box3(30.0, 30.0, 30.0)])), 0)
    A = fd.arrays()
    nu, pi = A["node"].view(np.uint32), A["prim"].view(np.int32)
    assert tuple(pi[p0, 0, :2]) == (3, 0)
    assert (nu[0, 3, 2], nu[0, 0, 0], nu[0, 0, 1]) == (F.CSG_DISCONTIGUOUS, 2, 1)
    assert nu[2, 3, 3] == 1                                  # the second sphere's transform
    assert tuple(pi[p1, 0, :2]) == (5, 3)
    assert nu[3, 0, 0] == 3                                  # tree root subNum: 3 tree nodes
    assert (nu[5, 3, 2], nu[5, 0, 0], nu[5, 0, 1]) == (F.CSG_OVERLAP, 2, 3)
    assert (nu[6, 3, 2], nu[7, 3, 2]) == (F.CSG_SPHERE, F.CSG_BOX3)


def test_contiguous_list_flags_more_than_eight_enters():
    # the reference keeps 8 enters per contiguous list (CSG/csg_intersect_node.h:460-470, undefined
    # beyond); the restatement drops the rest and raises the evaluator error flag
    fd = F.Foundry()
    chain = [F.translate(F.sphere(30.0), 0.0, 0.0, z) for z in np.arange(10) * 50.0]
    fd.add_prim(F.list_node("contiguous", chain), 0)
    A = fd.arrays()
    rays = np.array([[0.0], [0.0], [0.0], [0.0], [0.0], [1.0]], np.float32)       # inside the first: 9 enters
    out, err = O.csg_scan(A["node"], A["itra"], 0, rays, 0.0)
    assert err & 1
    rays = np.array([[0.0], [-100.0], [0.0], [0.0], [1.0], [0.0]], np.float32)     # across: 1 enter
    out, err = O.csg_scan(A["node"], A["itra"], 0, rays, 0.0)
    assert err == 0 and abs(out[0, 3] - 70.0) < 1e-3
