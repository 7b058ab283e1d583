"""CSGFoundry-layout geometry arrays built from Python.

The arrays have the byte layouts of the reference's persisted CSGFoundry
(CSG/CSGFoundry.cc:2769-2800 save, :2978-3016 load):

* ``node``  (Nn,4,4) float32  CSGNode   CSG/CSGNode.h:60-100 (q1.u.z boundary, q3.u.z typecode,
  q3.u.w gtransformIdx | complement<<31, q2/q3 bbox, root q0.u.x = subNum)
* ``prim``  (Np,4,4)          CSGPrim   CSG/CSGPrim.h:40-100 (q0.i numNode,nodeOffset,tranOffset,planOffset;
  q2/q3 bbox; q3.w globalPrimIdx)
* ``solid`` (Ns,3,4) int32    CSGSolid  CSG/CSGSolid.h:37-48 (label[16], numPrim, primOffset, type, intent, center_extent)
* ``inst``  (Ni,4,4) float32  qat4      sysrap/sqat4.h:345-389 (row-vector transform, identity ints in .w)
* ``itra``/``tran`` (Nt,4,4)  node transforms (inverse / forward)

so a foundry saved by the reference can be fed to the engine unchanged, and the synthetic
scenes here can be written out in the same format.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# typecodes sysrap/OpticksCSG.h
CSG_ZERO = 0
CSG_UNION = 1
CSG_INTERSECTION = 2
CSG_DIFFERENCE = 3
CSG_CONTIGUOUS = 11
CSG_DISCONTIGUOUS = 12
CSG_OVERLAP = 13
CSG_SPHERE = 101
CSG_ZSPHERE = 103
CSG_CYLINDER = 105
CSG_BOX3 = 110
CSG_TORUS = 116
CSG_SLAB = 106
CSG_CONE = 108
CSG_CONVEXPOLYHEDRON = 112
CSG_DISC = 113
CSG_HYPERBOLOID = 117
CSG_INFCYLINDER = 119
CSG_PHICUT = 121
CSG_HALFSPACE = 125
UNBOUNDED = 1.0e9     # box half-extent given to unbounded leaves (halfspace, slab, phicut, infcylinder)

OPS = {"union": CSG_UNION, "intersection": CSG_INTERSECTION, "difference": CSG_DIFFERENCE}
LISTS = {"contiguous": CSG_CONTIGUOUS, "discontiguous": CSG_DISCONTIGUOUS, "overlap": CSG_OVERLAP}


@dataclass
class Node:
    """One CSG node before serialisation; ``left``/``right`` only for operators."""
    typecode: int
    param: tuple = (0.0,) * 6
    left: "Node | None" = None
    right: "Node | None" = None
    transform: np.ndarray | None = None   # 4x4 row-vector (object -> parent frame)
    complement: bool = False
    bbox: tuple | None = None             # local (object frame) box of this leaf
    planes: np.ndarray | None = None      # convex polyhedron: (n,4) planes (unit normal, distance)
    subs: list | None = None              # list node: its leaves

    @property
    def is_leaf(self) -> bool:
        return self.typecode >= 100

    @property
    def is_list(self) -> bool:
        return CSG_CONTIGUOUS <= self.typecode <= CSG_OVERLAP


def sphere(r, center=(0.0, 0.0, 0.0)):
    cx, cy, cz = center
    return Node(CSG_SPHERE, (cx, cy, cz, r, 0.0, 0.0), bbox=(cx - r, cy - r, cz - r, cx + r, cy + r, cz + r))


def zsphere(r, z1, z2, center=(0.0, 0.0, 0.0)):
    """sphere radius r cut to z in [center.z+z1, center.z+z2] (zdelta in q1.xy)"""
    cx, cy, cz = center
    return Node(CSG_ZSPHERE, (cx, cy, cz, r, z1, z2), bbox=(cx - r, cy - r, cz + z1, cx + r, cy + r, cz + z2))


def cylinder(r, z1, z2):
    return Node(CSG_CYLINDER, (0.0, 0.0, 0.0, r, z1, z2), bbox=(-r, -r, z1, r, r, z2))


def box3(fx, fy, fz):
    return Node(CSG_BOX3, (fx, fy, fz, 0.0, 0.0, 0.0), bbox=(-fx / 2, -fy / 2, -fz / 2, fx / 2, fy / 2, fz / 2))


def torus(rmajor, rminor):
    """full-phi torus about z: param (rmin=0, rmax=rminor, rtor=rmajor, startPhi=0, deltaPhi=360)
    as sysrap/sn.h:3323-3337 sn::Torus stores it"""
    R, r = rmajor, rminor
    return Node(CSG_TORUS, (0.0, r, R, 0.0, 360.0, 0.0), bbox=(-(R + r), -(R + r), -r, R + r, R + r, r))


def cone(r1, z1, r2, z2):
    """cone frustum about z from radius r1 at z1 to r2 at z2 (z2 > z1), capped (CSGNode::Cone)"""
    R = max(r1, r2)
    return Node(CSG_CONE, (r1, z1, r2, z2, 0.0, 0.0), bbox=(-R, -R, z1, R, R, z2))


def hyperboloid(r0, zf, z1, z2):
    """one-sheet hyperboloid x^2+y^2 = r0^2((z/zf)^2+1) between z1 < z2, capped (CSGNode::Hyperboloid)"""
    R = r0 * math.sqrt((max(abs(z1), abs(z2)) / zf) ** 2 + 1.0)
    return Node(CSG_HYPERBOLOID, (r0, zf, z1, z2, 0.0, 0.0), bbox=(-R, -R, z1, R, R, z2))


def convexpolyhedron(planes, bbox):
    """intersection of half-spaces n.x <= w, planes (n,4) rows (nx, ny, nz, w) with unit normals"""
    pl = np.asarray(planes, dtype=np.float32).reshape(-1, 4)
    return Node(CSG_CONVEXPOLYHEDRON, (0.0,) * 6, bbox=tuple(bbox), planes=pl)


def cube_planes(h):
    """the six planes of the cube |x|,|y|,|z| <= h"""
    return [(1, 0, 0, h), (-1, 0, 0, h), (0, 1, 0, h), (0, -1, 0, h), (0, 0, 1, h), (0, 0, -1, h)]


def phicut(phi0, phi1):
    """wedge between the half-planes at azimuths phi0 < phi1 (radians) about z (CSGNode::PhiCut)"""
    U = UNBOUNDED
    return Node(CSG_PHICUT, (math.cos(phi0), math.sin(phi0), math.cos(phi1), math.sin(phi1), 0.0, 0.0),
                bbox=(-U, -U, -U, U, U, U))


def halfspace(n, w):
    """half-space n.x <= w (unit normal n)"""
    U = UNBOUNDED
    return Node(CSG_HALFSPACE, (n[0], n[1], n[2], w, 0.0, 0.0), bbox=(-U, -U, -U, U, U, U))


def slab(n, a, b):
    """slab a <= n.x <= b (unit normal n)"""
    U = UNBOUNDED
    return Node(CSG_SLAB, (n[0], n[1], n[2], 0.0, a, b), bbox=(-U, -U, -U, U, U, U))


def infcylinder(r):
    """cylinder of radius r about z, unbounded in z"""
    U = UNBOUNDED
    return Node(CSG_INFCYLINDER, (0.0, 0.0, 0.0, r, 0.0, 0.0), bbox=(-r, -r, -U, r, r, U))


def disc(inner, radius, z1, z2, cx=0.0, cy=0.0):
    """annulus inner < rho < radius about (cx, cy) between z1 < z2 (CSGNode::Disc)"""
    return Node(CSG_DISC, (cx, cy, inner, radius, z1, z2), bbox=(cx - radius, cy - radius, z1, cx + radius, cy + radius, z2))


def op(name, a: Node, b: Node) -> Node:
    return Node(OPS[name], left=a, right=b)


def list_node(kind: str, leaves) -> Node:
    """list node (CSGNode::ListHeader): "contiguous" (union of touching or overlapping leaves),
    "discontiguous" (union of disjoint leaves) or "overlap" (intersection of the leaves)"""
    return Node(LISTS[kind], subs=list(leaves))


def translate(n: Node, tx, ty, tz) -> Node:
    m = np.eye(4)
    m[3, :3] = (tx, ty, tz)
    n.transform = m if n.transform is None else n.transform @ m
    return n


def _height(n: Node) -> int:
    return 0 if n.is_leaf or n.is_list else 1 + max(_height(n.left), _height(n.right))


def _bbox_transformed(bb, m):
    if m is None:
        return bb
    pts = np.array([[bb[0 + 3 * (i & 1)], bb[1 + 3 * ((i >> 1) & 1)], bb[2 + 3 * ((i >> 2) & 1)], 1.0] for i in range(8)])
    w = pts @ m
    return tuple(w[:, :3].min(0)) + tuple(w[:, :3].max(0))


def _tree_bbox(n: Node):
    """bbox of a subtree in the frame of its parent (the node's own transform applied)"""
    if n.is_leaf:
        return _bbox_transformed(n.bbox, n.transform)
    if n.is_list:
        bbs = [_tree_bbox(c) for c in n.subs]
        if n.typecode == CSG_OVERLAP:
            bb = tuple(max(b[k] for b in bbs) for k in range(3)) + tuple(min(b[k] for b in bbs) for k in range(3, 6))
        else:
            bb = tuple(min(b[k] for b in bbs) for k in range(3)) + tuple(max(b[k] for b in bbs) for k in range(3, 6))
        return _bbox_transformed(bb, n.transform)
    a, b = _tree_bbox(n.left), _tree_bbox(n.right)
    if n.typecode == CSG_UNION:
        bb = tuple(min(a[k], b[k]) for k in range(3)) + tuple(max(a[k], b[k]) for k in range(3, 6))
    elif n.typecode == CSG_INTERSECTION:
        bb = tuple(max(a[k], b[k]) for k in range(3)) + tuple(min(a[k], b[k]) for k in range(3, 6))
    else:
        bb = a   # difference bounded by A
    return _bbox_transformed(bb, n.transform)


def _compose(local, parent):
    """row-vector transforms: a point takes ``local`` first, then ``parent``"""
    if local is None:
        return parent
    return local if parent is None else np.asarray(local) @ np.asarray(parent)


@dataclass
class Foundry:
    node: list = field(default_factory=list)
    prim: list = field(default_factory=list)
    solid: list = field(default_factory=list)
    inst: list = field(default_factory=list)
    tran: list = field(default_factory=list)
    itra: list = field(default_factory=list)
    plan: list = field(default_factory=list)

    # -------------------------------------------------------------- building
    def _add_transform(self, m) -> int:
        self.tran.append(np.asarray(m, dtype=np.float64))
        self.itra.append(np.linalg.inv(np.asarray(m, dtype=np.float64)))
        return len(self.tran)   # 1-based gtransformIdx

    def _node_row(self, n: Node | None, gm, boundary: int, index: int) -> np.ndarray:
        q = np.zeros((4, 4), dtype=np.float32)
        qu = q.view(np.uint32)
        if n is None:
            qu[3, 2] = CSG_ZERO
        else:
            if n.is_leaf:
                q[0, :4] = n.param[:4]
                q[1, :2] = n.param[4:6]
                if n.planes is not None:       # convex polyhedron: planeIdx, planeNum (CSG/CSGNode.h:204-207)
                    qu[0, 0] = len(self.plan)
                    qu[0, 1] = len(n.planes)
                    self.plan.extend(np.asarray(n.planes, np.float32))
                bb = n.bbox
            else:
                bb = _tree_bbox(n)
            q[2, 0:3] = bb[0:3]
            q[2, 3] = bb[3]
            q[3, 0:2] = bb[4:6]
            qu[3, 2] = n.typecode
            tidx = self._add_transform(gm) if (n.is_leaf and gm is not None) else 0
            qu[3, 3] = (tidx & 0x7FFFFFFF) | (0x80000000 if n.complement else 0)
        qu[1, 2] = boundary
        qu[1, 3] = index
        return q

    def add_prim(self, root: Node, boundary: int, mesh_idx: int = 0) -> int:
        """Serialise a tree as a complete binary tree (level order, CSG_ZERO padding), the leaves
        of its list nodes following it; a list at the root is its header then its leaves."""
        h = _height(root)
        num = (1 << (h + 1)) - 1
        slots: list[Node | None] = [None] * num

        gtran: list = [None] * num

        # a transform on an operator node moves its whole subtree: each leaf carries the product
        # of its own and its ancestors' transforms (the leaf's gtransform, as in CSG/CSGNode.h)
        def place(n, i, parent_m):
            slots[i] = n
            gtran[i] = _compose(n.transform, parent_m)
            if not n.is_leaf and not n.is_list:
                place(n.left, 2 * i + 1, gtran[i])
                place(n.right, 2 * i + 2, gtran[i])
        place(root, 0, None)
        offset = len(self.node)
        # list sub-nodes follow the tree; subOffset counts from the prim's first node
        # (CSG/CSGMaker.cc:800-860, CSG/csg_intersect_node.h:392-945)
        subs, cursor = [], num
        for i, n in enumerate(slots):
            if n is not None and n.is_list:
                subs.append((i, cursor))
                cursor += len(n.subs)
        for i, n in enumerate(slots):
            q = self._node_row(n, gtran[i], boundary, i)
            if n is not None and n.is_list:
                qu = q.view(np.uint32)
                qu[0, 0] = len(n.subs)
                qu[0, 1] = dict(subs)[i]
            self.node.append(q)
        for i, first in subs:
            for k, leaf in enumerate(slots[i].subs):
                if not leaf.is_leaf:
                    raise ValueError("list nodes hold leaves only")
                self.node.append(self._node_row(leaf, _compose(leaf.transform, gtran[i]), boundary, first + k))
        if not root.is_leaf and not root.is_list:
            self.node[offset].view(np.uint32)[0, 0] = num      # subNum: complete binary tree size
        bb = _tree_bbox(root)
        p = np.zeros((4, 4), dtype=np.float32)
        pi = p.view(np.int32)
        pi[0, 0] = cursor
        pi[0, 1] = offset
        pi[1, 1] = mesh_idx
        pi[1, 3] = len(self.prim)
        p[2, 0:3] = bb[0:3]
        p[2, 3] = bb[3]
        p[3, 0:2] = bb[4:6]
        pi[3, 3] = len(self.prim)       # globalPrimIdx
        self.prim.append(p)
        return len(self.prim) - 1

    def add_solid(self, label: str, prims: list[int]) -> int:
        assert prims == list(range(prims[0], prims[0] + len(prims))), "prims of a solid must be contiguous"
        s = np.zeros((3, 4), dtype=np.int32)
        lab = label.encode()[:16].ljust(16, b"\0")
        s[0, :] = np.frombuffer(lab, dtype=np.int32)
        s[1, 0] = len(prims)
        s[1, 1] = prims[0]
        self.solid.append(s)
        return len(self.solid) - 1

    def add_inst(self, m, gas_idx: int, sensor_identifier: int = -1, sensor_index: int = -1) -> int:
        """m : 4x4 row-vector object->world; sensor_identifier -1 means not a sensor (stored +1)"""
        q = np.asarray(m, dtype=np.float32).copy()
        qi = q.view(np.int32)
        ins = len(self.inst)
        qi[0, 3] = ins
        qi[1, 3] = gas_idx
        qi[2, 3] = sensor_identifier + 1
        qi[3, 3] = sensor_index
        self.inst.append(q)
        return ins

    # -------------------------------------------------------------- arrays
    def arrays(self) -> dict:
        def stack(lst, shape, dt):
            return np.ascontiguousarray(np.stack(lst).astype(dt)) if lst else np.zeros((0,) + shape, dtype=dt)
        return {
            "node": stack(self.node, (4, 4), np.float32),
            "prim": stack(self.prim, (4, 4), np.float32),
            "solid": stack(self.solid, (3, 4), np.int32),
            "inst": stack(self.inst, (4, 4), np.float32),
            "tran": stack([m.astype(np.float32) for m in self.tran], (4, 4), np.float32),
            "itra": stack([m.astype(np.float32) for m in self.itra], (4, 4), np.float32),
            "plan": stack(self.plan, (4,), np.float32),
        }

    def save(self, fold: str) -> None:
        """write the arrays as CSGFoundry/*.npy"""
        import os
        os.makedirs(fold, exist_ok=True)
        for k, v in self.arrays().items():
            np.save(os.path.join(fold, f"{k}.npy"), v)


def load_arrays(fold: str) -> dict:
    """read CSGFoundry/{node,prim,solid,inst,itra,plan}.npy as written by the reference"""
    import os
    out = {}
    for k in ("node", "prim", "solid", "inst", "itra", "plan", "tran"):
        p = os.path.join(fold, f"{k}.npy")
        if os.path.exists(p):
            out[k] = np.load(p)
    out.setdefault("plan", np.zeros((0, 4), dtype=np.float32))
    out.setdefault("itra", np.zeros((0, 4, 4), dtype=np.float32))
    return out


def look_at_z(pos, target) -> np.ndarray:
    """row-vector transform placing local +z along (target - pos), origin at pos"""
    pos = np.asarray(pos, dtype=np.float64)
    z = np.asarray(target, dtype=np.float64) - pos
    z /= np.linalg.norm(z)
    a = np.array([1.0, 0.0, 0.0]) if abs(z[0]) < 0.9 else np.array([0.0, 1.0, 0.0])
    x = np.cross(a, z)
    x /= np.linalg.norm(x)
    y = np.cross(z, x)
    m = np.eye(4)
    m[0, :3] = x
    m[1, :3] = y
    m[2, :3] = z
    m[3, :3] = pos
    return m


def fibonacci_sphere(n: int, radius: float) -> np.ndarray:
    i = np.arange(n, dtype=np.float64)
    z = 1.0 - 2.0 * (i + 0.5) / n
    r = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    ga = math.pi * (3.0 - math.sqrt(5.0))
    phi = ga * i
    return radius * np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=1)
