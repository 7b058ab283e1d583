"""Generate the committed golden fixtures under tests/golden/ from the reference's own code.

csg_scan_ref.npz : rays and the intersects computed by the reference's CSG intersector
                   (CSG/csg_intersect_tree.h etc. compiled for the CPU by oracle/Makefile `ref`
                   into oracle/_ref/libref_csg.so) for the benchmark tree without the torus
                   (the reference intersector has no torus leaf) and for each leaf alone.
csg_zoo_ref.npz  : the same for the further leaves (scenes.csg_leaf_zoo: cone, hyperboloid,
                   convexpolyhedron with its plan table, phicut, halfspace) through the reference's
                   tree intersector, and the slab / infcylinder / disc leaves one at a time through
                   the reference's own leaf functions (compiled there only under CSG_EXTRA).
csg_list_ref.npz : list nodes (scenes.csg_list_zoo: contiguous, discontiguous, overlap, and lists
                   inside boolean trees) through the reference's tree / list intersectors
                   (built WITH_CONTIGUOUS as its CSG library is).
planck_icdf_ref.npy : the black-body wavelength table QPlanck builds from sysrap/sblackbody.h
                   (oracle/_ref/libref_planck.so), 4096 float32.

Run from the repository root where the reference checkout is present:
    make -C oracle ref && python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from opticks_b200 import foundry as F  # noqa: E402
from opticks_b200 import scenes  # noqa: E402
from oracle import oracle as O  # noqa: E402


def leaf_foundry():
    fd = F.Foundry()
    prims = []
    for n in (F.sphere(240.0), F.zsphere(254.0, 0.0, 190.0), F.cylinder(250.0, -200.0, 200.0), F.box3(500.0, 500.0, 300.0)):
        prims.append(fd.add_prim(n, 0))
    # a complemented leaf and a transformed leaf inside small trees
    a = F.sphere(200.0)
    b = F.translate(F.box3(150.0, 150.0, 150.0), 50.0, -30.0, 120.0)
    prims.append(fd.add_prim(F.op("intersection", a, b), 0))
    c = F.cylinder(100.0, -300.0, 300.0)
    c.complement = True
    prims.append(fd.add_prim(F.op("intersection", F.sphere(250.0), c), 0))
    fd.add_solid("leaves", prims)
    fd.add_inst(np.eye(4), 0)
    return fd, prims


def main():
    out = {}
    fd, p = scenes.csg_scan_tree(with_torus=False)
    A = fd.arrays()
    rays = scenes.scan_rays(3000, seed=7, half=450.0)
    root = int(A["prim"].view(np.int32)[p, 0, 1])
    out["tree_node"] = A["node"]
    out["tree_itra"] = A["itra"] if len(A["itra"]) else np.zeros((1, 4, 4), np.float32)
    out["tree_root"] = np.int32(root)
    out["tree_rays"] = rays
    out["tree_isect"] = O.ref_csg_scan(A["node"], A["itra"], root, rays, 0.0)
    fd2, prims = leaf_foundry()
    B = fd2.arrays()
    out["leaf_node"] = B["node"]
    out["leaf_itra"] = B["itra"]
    out["leaf_roots"] = np.array([int(B["prim"].view(np.int32)[q, 0, 1]) for q in prims], np.int32)
    lr = scenes.scan_rays(1500, seed=11, half=400.0)
    out["leaf_rays"] = lr
    out["leaf_isect"] = np.stack([O.ref_csg_scan(B["node"], B["itra"], int(r), lr, 0.0) for r in out["leaf_roots"]])
    np.savez_compressed(os.path.join(ROOT, "tests", "golden", "csg_scan_ref.npz"), **out)
    print({k: getattr(v, "shape", v) for k, v in out.items()})
    zoo()
    lists()
    np.save(os.path.join(ROOT, "tests", "golden", "planck_icdf_ref.npy"), O.ref_planck_icdf())


def lists():
    fd, prims = scenes.csg_list_zoo()
    A = fd.arrays()
    rays = scenes.scan_rays(2000, seed=19, half=400.0)
    roots = np.array([int(A["prim"].view(np.int32)[p, 0, 1]) for p in prims], np.int32)
    out = {"node": A["node"], "itra": A["itra"], "plan": A["plan"], "prims": np.array(prims, np.int32),
           "roots": roots, "rays": rays}
    out["isect"] = np.stack([O.ref_csg_scan(A["node"], A["itra"], int(r), rays, 0.0, plan=A["plan"]) for r in roots])
    np.savez_compressed(os.path.join(ROOT, "tests", "golden", "csg_list_ref.npz"), **out)
    print({k: getattr(v, "shape", v) for k, v in out.items()})


EXTRA_LEAVES = (F.slab((0.6, 0.8, 0.0), -100.0, 150.0), F.infcylinder(120.0),
                F.disc(50.0, 250.0, -10.0, 10.0), F.disc(0.0, 230.0, -5.0, 5.0, 20.0, -30.0))


def zoo():
    fd, prims = scenes.csg_leaf_zoo()
    A = fd.arrays()
    rays = scenes.scan_rays(2000, seed=13, half=400.0)
    keep = [p for k, p in enumerate(prims) if k not in scenes.ZOO_EXTRA_PRIMS]
    roots = np.array([int(A["prim"].view(np.int32)[p, 0, 1]) for p in keep], np.int32)
    out = {"node": A["node"], "itra": A["itra"], "plan": A["plan"], "prims": np.array(keep, np.int32),
           "roots": roots, "rays": rays}
    out["isect"] = np.stack([O.ref_csg_scan(A["node"], A["itra"], int(r), rays, 0.0, plan=A["plan"]) for r in roots])
    fe = F.Foundry()
    ep = [fe.add_prim(n, 0) for n in EXTRA_LEAVES]
    B = fe.arrays()
    q = np.stack([B["node"][int(B["prim"].view(np.int32)[p, 0, 1])].reshape(-1)[:8] for p in ep])
    tc = np.array([int(B["node"].view(np.uint32)[int(B["prim"].view(np.int32)[p, 0, 1]), 3, 2]) for p in ep], np.int32)
    out["extra_q"] = q
    out["extra_typecode"] = tc
    out["extra_isect"] = np.stack([O.ref_leaf_extra_scan(int(t), qq, rays) for t, qq in zip(tc, q)])
    np.savez_compressed(os.path.join(ROOT, "tests", "golden", "csg_zoo_ref.npz"), **out)
    print({k: getattr(v, "shape", v) for k, v in out.items()})


if __name__ == "__main__":
    main()
