"""Writes tests/golden/npfold/: a CSGFoundry directory and its SSim/stree/standard arrays written by
the reference's own array writer (sysrap/NP.hh, through oracle/_ref/libref_npfold.so, built by
`make -C oracle ref` from the reference checkout), for the loader tests.

The geometry is the leaf-zoo box (a detecting box with acrylic bodies made of cones, hyperboloids,
convexpolyhedra with their plan rows, phicut and halfspace cuts), the physics its boundary library
plus the detector's scintillation ICDF.  Run from the repository root:

    python tests/golden/make_npfold.py
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from opticks_b200 import material as M  # noqa: E402
from opticks_b200 import scenes  # noqa: E402

OUT = os.path.join(HERE, "npfold", "CSGFoundry")


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def fixture_scene():
    """the arrays the fixture holds, as the engine takes them"""
    fd, lib, _, _ = scenes.leaf_zoo_detector(1)
    geom = fd.arrays()
    phys = lib.arrays()
    phys["icdf"] = M.gaussian_icdf(430.0, 20.0)
    names = ["/".join(b) for b in lib.boundaries]
    return geom, phys, names


def main():
    L = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_npfold.so"))
    L.ref_write_foundry.restype = C.c_int
    L.ref_write_standard.restype = C.c_int
    geom, phys, names = fixture_scene()
    os.makedirs(OUT, exist_ok=True)
    g = {k: np.ascontiguousarray(geom[k]) for k in ("solid", "prim", "node", "itra", "inst", "plan")}
    tran = np.ascontiguousarray(np.linalg.inv(g["itra"].astype(np.float64)).astype(np.float32)) if len(g["itra"]) else g["itra"]
    meshnames = "\n".join(f"zoo_{k}" for k in range(len(g["prim"]))).encode()
    rc = L.ref_write_foundry(OUT.encode(), _p(g["solid"].astype(np.int32)), len(g["solid"]), _p(g["prim"]), len(g["prim"]),
                             _p(g["node"]), len(g["node"]), _p(tran), len(tran), _p(g["itra"]), len(g["itra"]),
                             _p(g["inst"]), len(g["inst"]), _p(g["plan"].astype(np.float32)), len(g["plan"]), meshnames)
    assert rc == 0, rc
    std = os.path.join(OUT, "SSim", "stree", "standard")
    os.makedirs(std, exist_ok=True)
    bnd = np.ascontiguousarray(phys["bnd"], np.float64)
    opt = np.ascontiguousarray(phys["optical"].reshape(-1, 4, 4).view(np.int32))
    icdf = np.ascontiguousarray(phys["icdf"], np.float64)
    rc = L.ref_write_standard(std.encode(), _p(bnd), bnd.shape[0], bnd.shape[3], "\n".join(names).encode(), _p(opt), _p(icdf),
                              icdf.shape[0], icdf.shape[1], icdf.shape[2], C.c_float(60.0), C.c_float(820.0), C.c_float(1.0))
    assert rc == 0, rc
    print("wrote", OUT)


if __name__ == "__main__":
    main()
