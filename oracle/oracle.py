"""ctypes access to the checkers under oracle/ — TEST INFRASTRUCTURE ONLY.

* ``liboracle.so``        C restatement of the simulate path (oracle.c) : CPU, FP32 + FP64 CSG
* ``_ref/libref_csg.so``  the reference's own CSG intersector compiled for the CPU
* ``_ref/libref_sim.so``  the reference's own qsim/CSG device code driven on the GPU
* ``_ref/libref_spm.so``  the reference's own hit merge (sysrap/SPM.cu) on the GPU
* ``_ref/libref_cpu_sim.so`` the reference's own qsim/CSG path compiled for the CPU (MOCK_CURAND)
* ``_ref/libref_npfold.so`` arrays written by the reference's own NP.hh (loader fixtures)
* ``merge.py``            numpy restatement of the hit merge

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this module, and
only as the checker / the timed CPU baseline.  Nothing in opticks_b200/ imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_CSG = os.path.join(HERE, "_ref", "libref_csg.so")
REF_SIM = os.path.join(HERE, "_ref", "libref_sim.so")
REF_PLANCK = os.path.join(HERE, "_ref", "libref_planck.so")
REF_SPM = os.path.join(HERE, "_ref", "libref_spm.so")


def build(ref: bool = False) -> None:
    """make liboracle.so (and the reference builds when the reference checkout is present)"""
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
    if ref and subprocess.run(["make", "-s", "-C", HERE, "ref-present"]).returncode == 0:
        subprocess.run(["make", "-s", "-C", HERE, "ref"], check=True)


class OracleScene(C.Structure):
    _fields_ = [
        ("node", C.c_void_p), ("itra", C.c_void_p), ("inst_inv", C.c_void_p),
        ("pair_inst", C.c_void_p), ("pair_node", C.c_void_p), ("pair_gpbd", C.c_void_p), ("pair_iiid", C.c_void_p),
        ("num_pair", C.c_int),
        ("bnd", C.c_void_p), ("bnd_w", C.c_int), ("bnd_h", C.c_int), ("nm0", C.c_float), ("nms", C.c_float),
        ("optical", C.c_void_p), ("icdf", C.c_void_p), ("icdf_w", C.c_int), ("icdf_h", C.c_int), ("hd_factor", C.c_int),
        ("max_bounce", C.c_int), ("max_time", C.c_float), ("tmin", C.c_float), ("tmin0", C.c_float),
        ("eps0_mask", C.c_uint), ("hit_mask", C.c_uint), ("polish", C.c_int),
        ("pair_bbox", C.c_void_p), ("plan", C.c_void_p), ("input_photon", C.c_void_p), ("num_input", C.c_longlong),
        ("planck", C.c_void_p),
    ]


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        L.oracle_simulate.restype = C.c_int
        L.oracle_simulate.argtypes = [C.POINTER(OracleScene), C.c_void_p, C.c_int, C.c_longlong, C.c_longlong,
                                      C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
        L.oracle_csg_scan.restype = C.c_int
        L.oracle_csg_scan.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_float, C.c_void_p, C.c_longlong,
                                      C.c_void_p, C.c_int, C.c_int]
        L.oracle_csg_scan_t64.restype = C.c_int
        L.oracle_csg_scan_t64.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_float, C.c_void_p, C.c_longlong,
                                          C.c_void_p]
        L.oracle_csg_scan_t64d.restype = C.c_int
        L.oracle_csg_scan_t64d.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_double, C.c_void_p, C.c_longlong,
                                           C.c_void_p]
        L.oracle_csg_action.restype = C.c_int
        L.oracle_csg_action.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int]
        L.oracle_tex2d_f1.restype = C.c_float
        L.oracle_tex2d_f1.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_float]
        L.oracle_tex2d_f4.restype = None
        L.oracle_tex2d_f4.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_float, C.c_void_p]
        L.oracle_threads.restype = C.c_int
        L.oracle_adjoint.restype = C.c_int
        L.oracle_adjoint.argtypes = [C.POINTER(OracleScene), C.c_void_p, C.c_int, C.c_longlong, C.c_longlong, C.c_void_p, C.c_int,
                                     C.c_uint, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, C.c_void_p, C.c_void_p]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def instance_pairs(geom: dict):
    """(instance, prim) pairs in instance order with the IS/CH identity words, and world->object
    inverses of the instance transforms (computed in double, stored float32)"""
    node, prim, solid, inst = geom["node"], geom["prim"], geom["solid"], geom["inst"]
    nu = node.view(np.uint32)
    pi = prim.view(np.int32)
    ii = inst.view(np.int32)
    inv = np.zeros((len(inst), 4, 4), np.float32)
    pin, pnode, pgb, pid = [], [], [], []
    for i in range(len(inst)):
        m = inst[i].astype(np.float64).copy()
        m[:3, 3] = 0.0
        m[3, 3] = 1.0
        inv[i] = np.linalg.inv(m).astype(np.float32)
        inv[i][:3, 3] = 0.0
        inv[i][3, 3] = 1.0
        gas = ii[i, 1, 3]
        sid1 = ii[i, 2, 3]
        num, off = solid[gas, 1, 0], solid[gas, 1, 1]
        for p in range(off, off + num):
            no = pi[p, 0, 1]
            gpi = pi[p, 3, 3]
            bnd = nu[no, 1, 2]
            pin.append(i)
            pnode.append(no)
            pgb.append(((gpi & 0xFFFF) << 16) | (bnd & 0xFFFF))
            pid.append(((i & 0xFFFF) << 16) | (sid1 & 0xFFFF))
    return (inv, np.array(pin, np.int32), np.array(pnode, np.int32), np.array(pgb, np.uint32), np.array(pid, np.uint32))


def pair_world_boxes(geom: dict, pin, pnode) -> np.ndarray:
    """padded world AABB of each (instance, prim) pair from the CSGPrim box (q2,q3) and the
    instance transform, in double; only used to skip hopeless pairs in the brute-force loop"""
    prim, inst = geom["prim"], geom["inst"]
    pi = prim.view(np.int32)
    root_to_prim = {int(pi[p, 0, 1]): p for p in range(len(prim))}
    out = np.zeros((len(pin), 6), np.float32)
    for k, (i, no) in enumerate(zip(pin, pnode)):
        p = root_to_prim[int(no)]
        bb = np.array([prim[p, 2, 0], prim[p, 2, 1], prim[p, 2, 2], prim[p, 2, 3], prim[p, 3, 0], prim[p, 3, 1]], np.float64)
        m = inst[i].astype(np.float64).copy()
        m[:3, 3] = 0.0
        m[3, 3] = 1.0
        c = np.array([[bb[0 + 3 * (j & 1)], bb[1 + 3 * ((j >> 1) & 1)], bb[2 + 3 * ((j >> 2) & 1)], 1.0] for j in range(8)])
        w = (c @ m)[:, :3]
        lo, hi = w.min(0), w.max(0)
        pad = 1e-3 * (hi - lo).max() + 1e-5 * np.abs(w).max() + 1e-2
        out[k, :3] = lo - pad
        out[k, 3:] = hi + pad
    return out


def planck_icdf() -> np.ndarray:
    """the oracle's restatement of QPlanck's black-body wavelength ICDF (4096 float32)"""
    out = np.zeros(4096, np.float32)
    L = lib()
    L.oracle_planck_icdf.restype = C.c_int
    L.oracle_planck_icdf.argtypes = [C.c_void_p, C.c_int]
    if L.oracle_planck_icdf(_p(out), 4096) != 0:
        raise RuntimeError("oracle_planck_icdf failed")
    return out


def have_ref_planck() -> bool:
    return os.path.exists(REF_PLANCK)


def ref_planck_icdf() -> np.ndarray:
    """the reference's own table (sysrap/sblackbody.h compiled on the CPU)"""
    L = C.CDLL(REF_PLANCK)
    L.ref_planck_icdf.restype = C.c_int
    L.ref_planck_icdf.argtypes = [C.c_void_p, C.c_int]
    out = np.zeros(4096, np.float32)
    if L.ref_planck_icdf(_p(out), 4096) != 0:
        raise RuntimeError("ref_planck_icdf failed")
    return out


class Scene:
    """keeps the arrays alive behind an OracleScene"""

    def __init__(self, geom: dict, phys: dict, max_bounce=31, max_time=1e27, tmin=0.05, tmin0=0.05,
                 eps0_mask=0x4 | 0x1 | 0x2 | 0x20 | 0x10, hit_mask=0x40, polish=0, cull=True, input_photon=None):
        self.node = np.ascontiguousarray(geom["node"], np.float32)
        itra = geom.get("itra")
        self.itra = np.ascontiguousarray(itra if itra is not None and len(itra) else np.zeros((1, 4, 4)), np.float32)
        self.inst_inv, self.pin, self.pnode, self.pgb, self.pid = instance_pairs(geom)
        self.bnd = np.ascontiguousarray(phys["bnd"], np.float32)
        self.optical = np.ascontiguousarray(phys["optical"], np.uint32)
        icdf = phys.get("icdf")
        self.icdf = None if icdf is None else np.ascontiguousarray(icdf, np.float32)
        nb, nwl = self.bnd.shape[0], self.bnd.shape[3]
        self.pair_bbox = pair_world_boxes(geom, self.pin, self.pnode) if cull else None
        self.plan = _plan(geom.get("plan"))
        self.s = OracleScene(
            _p(self.node), _p(self.itra), _p(self.inst_inv), _p(self.pin), _p(self.pnode), _p(self.pgb), _p(self.pid),
            len(self.pin), _p(self.bnd), nwl, nb * 8, float(phys.get("wl_low", 60.0)), float(phys.get("wl_step", 1.0)),
            _p(self.optical), _p(self.icdf), 0 if self.icdf is None else self.icdf.shape[1],
            0 if self.icdf is None else self.icdf.shape[0], int(phys.get("hd_factor", 20)),
            max_bounce, max_time, tmin, tmin0, eps0_mask, hit_mask, polish, _p(self.pair_bbox), _p(self.plan),
            None, 0, None)
        self.planck = planck_icdf()
        self.s.planck = _p(self.planck)
        self.input_photon = None
        if input_photon is not None:
            self.input_photon = np.ascontiguousarray(input_photon, np.float32).reshape(-1, 4, 4)
            self.s.input_photon = _p(self.input_photon)
            self.s.num_input = len(self.input_photon)

    def simulate(self, gs: np.ndarray, uniforms: np.ndarray, first: int = 0):
        gs = np.ascontiguousarray(gs, np.float32).reshape(-1, 6, 4)
        u = np.ascontiguousarray(uniforms, np.float32)
        n, K = u.shape
        photon = np.zeros((n, 4, 4), np.float32)
        seq = np.zeros((n, 2, 2), np.uint64)
        err = lib().oracle_simulate(C.byref(self.s), _p(gs), len(gs), first, n, _p(u), K, _p(photon), _p(seq))
        return photon, seq, err

    def adjoint(self, gs: np.ndarray, uniforms: np.ndarray, mat_line: int, wl_lo: float, wl_hi: float, num_sensor: int,
                first: int = 0, wl_low: float = 60.0, wl_step: float = 1.0):
        """FP64 reference of the score-function estimator (the scene's tables must already hold theta)"""
        gs = np.ascontiguousarray(gs, np.float32).reshape(-1, 6, 4)
        u = np.ascontiguousarray(uniforms, np.float32)
        n, K = u.shape
        mat = int(self.optical[mat_line, 0])
        hits = np.zeros((num_sensor,), np.float64)
        grad = np.zeros((num_sensor, 32), np.float64)
        err = lib().oracle_adjoint(C.byref(self.s), _p(gs), len(gs), first, n, _p(u), K, mat, wl_low, wl_step, wl_lo,
                                   (wl_hi - wl_lo) / 8.0, num_sensor, _p(hits), _p(grad))
        return hits, grad, err


def _plan(plan):
    return np.ascontiguousarray(plan if plan is not None and len(plan) else np.zeros((1, 4)), np.float32)


def csg_scan(node, itra, root: int, rays: np.ndarray, tmin: float = 0.0, use_double: bool = False, polish: bool = False,
             plan=None):
    node = np.ascontiguousarray(node, np.float32)
    itra = np.ascontiguousarray(itra if itra is not None and len(itra) else np.zeros((1, 4, 4)), np.float32)
    pl = _plan(plan)
    rays = np.ascontiguousarray(rays, np.float32)
    n = rays.shape[1]
    out = np.zeros((n, 4), np.float32)
    err = lib().oracle_csg_scan(_p(node), _p(itra), _p(pl), root, tmin, _p(rays), n, _p(out), int(use_double), int(polish))
    return out, err


def csg_scan_t64(node, itra, root: int, rays: np.ndarray, tmin: float = 0.0, plan=None):
    node = np.ascontiguousarray(node, np.float32)
    itra = np.ascontiguousarray(itra if itra is not None and len(itra) else np.zeros((1, 4, 4)), np.float32)
    pl = _plan(plan)
    rays = np.ascontiguousarray(rays, np.float32)
    n = rays.shape[1]
    t = np.zeros((n,), np.float64)
    err = lib().oracle_csg_scan_t64(_p(node), _p(itra), _p(pl), root, tmin, _p(rays), n, _p(t))
    return t, err


def csg_scan_t64d(node, itra, root: int, rays64: np.ndarray, tmin: float = 0.0, plan=None):
    """FP64 distances of FP64 rays (SoA (6,n) float64) against one prim; 0 for a miss"""
    node = np.ascontiguousarray(node, np.float32)
    itra = np.ascontiguousarray(itra if itra is not None and len(itra) else np.zeros((1, 4, 4)), np.float32)
    pl = _plan(plan)
    rays64 = np.ascontiguousarray(rays64, np.float64)
    n = rays64.shape[1]
    t = np.zeros((n,), np.float64)
    err = lib().oracle_csg_scan_t64d(_p(node), _p(itra), _p(pl), root, tmin, _p(rays64), n, _p(t))
    return t, err


def trace_t64(geom: dict, rays: np.ndarray, inst_idx: np.ndarray, prim_idx: np.ndarray, tmin: float = 0.0) -> np.ndarray:
    """FP64 distance along each world ray (SoA (6,n) float32) to the given (instance, prim): the ray is
    carried into the prim's frame in double (row-vector qat4 convention, identity words in the .w
    column zeroed) and intersected with the FP64 CSG evaluator; 0 where it misses that prim"""
    inst = geom["inst"].astype(np.float64)
    prim = geom["prim"]
    pi = prim.view(np.int32)
    n = rays.shape[1]
    t = np.zeros(n, np.float64)
    o = np.c_[rays[:3].T.astype(np.float64), np.ones(n)]
    d = np.c_[rays[3:].T.astype(np.float64), np.zeros(n)]
    m = inst.copy()
    m[:, :3, 3] = 0.0
    m[:, 3, 3] = 1.0
    inv = np.linalg.inv(m)[inst_idx]
    lo = np.einsum("ni,nij->nj", o, inv)[:, :3]
    ld = np.einsum("ni,nij->nj", d, inv)[:, :3]
    for p in np.unique(prim_idx):
        sel = np.nonzero(prim_idx == p)[0]
        r64 = np.ascontiguousarray(np.concatenate([lo[sel].T, ld[sel].T]))
        t[sel], _ = csg_scan_t64d(geom["node"], geom.get("itra"), int(pi[p, 0, 1]), r64, tmin, plan=geom.get("plan"))
    return t


def tex2d_f1(data: np.ndarray, x: float, y: float) -> float:
    d = np.ascontiguousarray(data, np.float32)
    H, W = d.shape[:2]
    return lib().oracle_tex2d_f1(_p(d), W, H, x, y)


# ---------------------------------------------------------------- reference builds
def have_ref_csg() -> bool:
    return os.path.exists(REF_CSG)


def have_ref_sim() -> bool:
    return os.path.exists(REF_SIM)


REF_CPU_SIM = os.path.join(HERE, "_ref", "libref_cpu_sim.so")


def have_ref_cpu_sim() -> bool:
    return os.path.exists(REF_CPU_SIM)


def ref_simulate_cpu(geom: dict, phys: dict, gs: np.ndarray, nthreads: int = 0, seed: int = 1, max_bounce: int = 31,
                     max_time: float = 1e27, tmin: float = 0.05, tmin0: float = 0.05,
                     eps0_mask: int = 0x4 | 0x1 | 0x2 | 0x20 | 0x10, outputs: bool = True):
    """the reference's qsim/CSG path compiled for the CPU (ref_cpu_sim.cc): its own generation and
    propagation with its CPU random generator (mt19937_64 per thread, so not the GPU streams) and
    its nearest-sample mock textures; returns (photon (N,4,4), seq (N,2,2), seconds, threads)"""
    L = C.CDLL(REF_CPU_SIM)
    f = L.ref_cpu_sim_run
    f.restype = C.c_int
    f.argtypes = [C.c_void_p] * 4 + [C.c_void_p] * 5 + [C.c_int] + [C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_float, C.c_void_p] + \
                 [C.c_void_p, C.c_int, C.c_int, C.c_int] + [C.c_void_p, C.c_int, C.c_longlong, C.c_int, C.c_float, C.c_float, C.c_float,
                                                            C.c_uint] + \
                 [C.c_ulonglong, C.c_int, C.c_void_p, C.c_void_p, C.POINTER(C.c_double)]
    node = np.ascontiguousarray(geom["node"], np.float32)
    itra = geom.get("itra")
    itra = np.ascontiguousarray(itra if itra is not None and len(itra) else np.zeros((1, 4, 4)), np.float32)
    pl = _plan(geom.get("plan"))
    inv, pin, pnode, pgb, pid = instance_pairs(geom)
    bbox = np.ascontiguousarray(pair_world_boxes(geom, pin, pnode), np.float32)
    bnd = np.ascontiguousarray(phys["bnd"], np.float32)
    optical = np.ascontiguousarray(phys["optical"], np.uint32)
    icdf = phys.get("icdf")
    icdf = None if icdf is None else np.ascontiguousarray(icdf, np.float32)
    gs = np.ascontiguousarray(gs, np.float32).reshape(-1, 6, 4)
    N = int(gs.view(np.int32)[:, 0, 3].clip(0).sum())
    photon = np.zeros((N, 4, 4), np.float32) if outputs else None
    seq = np.zeros((N, 2, 2), np.uint64) if outputs else None
    secs = C.c_double(0.0)
    nt = f(_p(node), _p(itra), _p(pl), _p(inv), _p(pin), _p(pnode), _p(pgb), _p(pid), _p(bbox), len(pin),
           _p(bnd), bnd.shape[0], bnd.shape[3], float(phys.get("wl_low", 60.0)), float(phys.get("wl_step", 1.0)), _p(optical),
           _p(icdf), 0 if icdf is None else icdf.shape[1], 0 if icdf is None else icdf.shape[0], int(phys.get("hd_factor", 20)),
           _p(gs), len(gs), N, max_bounce, max_time, tmin, tmin0, eps0_mask, seed, nthreads, _p(photon), _p(seq), C.byref(secs))
    if nt < 0:
        raise RuntimeError(f"ref_cpu_sim_run failed {nt}")
    return photon, seq, secs.value, nt


def have_ref_spm() -> bool:
    return os.path.exists(REF_SPM)


def ref_merge_gpu(records: np.ndarray, select_flagmask: int = 0xFFFFFFFF, time_window: float = 1.0) -> np.ndarray:
    """SPM::merge_partial_select of the reference on the GPU (sphoton (n,4,4) or sphotonlite (n,4))"""
    L = C.CDLL(REF_SPM)
    L.ref_spm_merge.restype = C.c_int
    L.ref_spm_merge.argtypes = [C.c_void_p, C.c_longlong, C.c_int, C.c_uint, C.c_float, C.c_void_p, C.c_longlong,
                                C.POINTER(C.c_longlong)]
    rec = np.ascontiguousarray(records)
    lite = 1 if rec.ndim == 2 else 0
    out = np.zeros_like(rec)
    no = C.c_longlong(0)
    rc = L.ref_spm_merge(_p(rec), len(rec), lite, select_flagmask & 0xFFFFFFFF, time_window, _p(out), len(rec), C.byref(no))
    if rc != 0:
        raise RuntimeError(f"ref_spm_merge failed {rc}")
    return out[: no.value]


def ref_csg_scan(node, itra, root: int, rays: np.ndarray, tmin: float = 0.0, nthread: int = 0, plan=None):
    L = C.CDLL(REF_CSG)
    L.ref_csg_scan.restype = C.c_int
    L.ref_csg_scan.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_float, C.c_void_p, C.c_longlong, C.c_void_p,
                               C.c_int]
    node = np.ascontiguousarray(node, np.float32)
    itra = np.ascontiguousarray(itra if itra is not None and len(itra) else np.zeros((1, 4, 4)), np.float32)
    pl = _plan(plan)
    rays = np.ascontiguousarray(rays, np.float32)
    n = rays.shape[1]
    out = np.zeros((n, 4), np.float32)
    L.ref_csg_scan(_p(node), _p(itra), _p(pl), root, tmin, _p(rays), n, _p(out), nthread or (os.cpu_count() or 1))
    return out


def ref_leaf_extra_scan(typecode: int, q0q1, rays: np.ndarray, tmin: float = 0.0):
    """one slab / infcylinder / disc leaf through the reference's own leaf function (CPU)"""
    L = C.CDLL(REF_CSG)
    L.ref_leaf_extra_scan.restype = C.c_int
    L.ref_leaf_extra_scan.argtypes = [C.c_int, C.c_void_p, C.c_float, C.c_void_p, C.c_longlong, C.c_void_p]
    q = np.ascontiguousarray(np.asarray(q0q1, np.float32).reshape(8))
    rays = np.ascontiguousarray(rays, np.float32)
    n = rays.shape[1]
    out = np.zeros((n, 4), np.float32)
    if L.ref_leaf_extra_scan(typecode, _p(q), tmin, _p(rays), n, _p(out)) != 0:
        raise ValueError(f"typecode {typecode} is not a slab, infcylinder or disc")
    return out


def ref_scan_gpu(node, itra, root: int, rays: np.ndarray, tmin: float = 0.0, plan=None):
    L = C.CDLL(REF_SIM)
    L.ref_scan_run.restype = C.c_int
    L.ref_scan_run.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_void_p,
                               C.c_longlong, C.c_void_p]
    node = np.ascontiguousarray(node, np.float32)
    itra = np.ascontiguousarray(itra if itra is not None and len(itra) else np.zeros((1, 4, 4)), np.float32)
    rays = np.ascontiguousarray(rays, np.float32)
    n = rays.shape[1]
    out = np.zeros((n, 4), np.float32)
    pl = _plan(plan)
    rc = L.ref_scan_run(_p(node), len(node), _p(itra), len(itra), _p(pl), len(pl), root, tmin, _p(rays), n, _p(out))
    if rc != 0:
        raise RuntimeError(f"ref_scan_run failed {rc}")
    return out


# gencodes the driver gives the reference's qsim::generate_photon everything for
# (qudarap/qsim.h:2532-2561): torch, carrier, Cerenkov, scintillation, and input photons when given
REF_GENCODES = (6, 14, 15, 16, 19)
# torch types the reference's storch::generate fills a photon for (sysrap/storchtype.h:8-18,
# sysrap/storch.h:207-470): disc, line, point, circle, rectangle, sphere_marsaglia, sphere
REF_TORCH_TYPES = range(1, 8)


def ref_genstep_check(gs: np.ndarray, have_input: bool = False) -> None:
    """refuse gensteps the reference's device code is not given the means to generate: a torch
    genstep of a type storch::generate does not fill leaves the photon unset (zero wavelength
    then samples the Planck texture, qudarap/qsim.h:2541-2544, which this driver sets up as
    QPlanck does); input photons need the input array"""
    gi = gs.view(np.int32)
    for k in range(len(gs)):
        code = int(gi[k, 0, 0])
        if code not in REF_GENCODES:
            raise ValueError(f"genstep {k}: gencode {code} is not one the reference driver generates")
        if code == 19 and not have_input:
            raise ValueError(f"genstep {k}: INPUT_PHOTON genstep without input photons")
        if code == 6 and int(gi[k, 5, 3]) not in REF_TORCH_TYPES:
            raise ValueError(f"genstep {k}: torch type {int(gi[k, 5, 3])} is not a reference torch type")


def ref_simulate_gpu(geom: dict, phys: dict, gs: np.ndarray, event_index: int = 0, seed: int = 0, skip: int = 100000,
                     max_bounce: int = 31, max_time: float = 1e27, tmin: float = 0.05, tmin0: float = 0.05,
                     eps0_mask: int = 0x4 | 0x1 | 0x2 | 0x20 | 0x10, record: bool = False, input_photon=None):
    """run the reference's qsim on the GPU through ref_sim.cu; returns photon (N,4,4), seq (N,2,2)
    and, with ``record``, the per-point sphoton records (N,max_bounce+1,4,4) and per-trace prd
    (N,max_bounce+1,2,4) that the reference's sctx::point / sctx::trace write"""
    L = C.CDLL(REF_SIM)
    f = L.ref_sim_run
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                  C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                  C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_float, C.c_void_p,
                  C.c_void_p, C.c_int, C.c_int, C.c_int,
                  C.c_ulonglong, C.c_ulonglong, C.c_int,
                  C.c_void_p, C.c_int, C.c_longlong,
                  C.c_int, C.c_float, C.c_float, C.c_float, C.c_uint,
                  C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_longlong]
    node = np.ascontiguousarray(geom["node"], np.float32)
    itra = geom.get("itra")
    itra = np.ascontiguousarray(itra if itra is not None and len(itra) else np.zeros((1, 4, 4)), np.float32)
    inv, pin, pnode, pgb, pid = instance_pairs(geom)
    bnd = np.ascontiguousarray(phys["bnd"], np.float32)
    optical = np.ascontiguousarray(phys["optical"], np.uint32)
    icdf = phys.get("icdf")
    icdf = None if icdf is None else np.ascontiguousarray(icdf, np.float32)
    gs = np.ascontiguousarray(gs, np.float32).reshape(-1, 6, 4)
    inp = None if input_photon is None else np.ascontiguousarray(input_photon, np.float32).reshape(-1, 4, 4)
    ref_genstep_check(gs, inp is not None)
    N = int(gs.view(np.int32)[:, 0, 3].clip(0).sum())
    photon = np.zeros((N, 4, 4), np.float32)
    seq = np.zeros((N, 2, 2), np.uint64)
    max_record = max_bounce + 1 if record else 0
    rec = np.zeros((N, max_record, 4, 4), np.float32) if record else None
    prd = np.zeros((N, max_record, 2, 4), np.float32) if record else None
    pl = _plan(geom.get("plan"))
    rc = f(_p(node), len(node), _p(itra), len(itra), _p(pl), len(pl), _p(inv), len(inv), _p(pin), _p(pnode), _p(pgb), _p(pid),
           len(pin),
           _p(bnd), bnd.shape[0], bnd.shape[3], float(phys.get("wl_low", 60.0)), float(phys.get("wl_step", 1.0)), _p(optical),
           _p(icdf), 0 if icdf is None else icdf.shape[1], 0 if icdf is None else icdf.shape[0], int(phys.get("hd_factor", 20)),
           seed, skip, event_index, _p(gs), len(gs), N, max_bounce, max_time, tmin, tmin0, eps0_mask, _p(photon), _p(seq),
           _p(rec) if record else None, _p(prd) if record else None, max_record, _p(inp), 0 if inp is None else len(inp))
    if rc != 0:
        raise RuntimeError(f"ref_sim_run failed {rc}")
    return (photon, seq, rec, prd) if record else (photon, seq)
