"""Reading and writing the reference's on-disk geometry and material arrays.

A reference geometry directory (``$HOME/.opticks/GEOM/<GEOM>/CSGFoundry``) holds the CSGFoundry
arrays that ``CSGFoundry::load`` reads (CSG/CSGFoundry.cc:2978-3016): ``solid.npy``, ``prim.npy``,
``node.npy``, ``tran.npy``, ``itra.npy``, ``inst.npy``, the optional ``plan.npy``, and the names
``meshname.txt`` / ``mmlabel.txt`` with ``meta.txt``.  Beside them, ``SSim/stree/standard`` holds
the material/surface arrays the reference uploads (sysrap/snam.h:15-17): ``bnd.npy``
(num_bnd, 4, 2, num_wl, 4) with its wavelength domain in the sidecar ``bnd_meta.txt``
(``domain_low``/``domain_high``/``domain_step``, key:value lines, sysrap/sstandard.h:503-505,
the NP ``<name>_meta.txt`` convention), ``bnd_names.txt``, ``optical.npy`` (num_bnd*4, 4) uint32 and
``icdf.npy`` (3, 4096, 1) (qudarap/QScint.cc:84-120).

``load_geom(cfbase)`` returns the (geometry, physics) dicts ``engine.Engine`` takes;
``save_geom`` writes the same layout, so arrays built with ``foundry``/``material`` can be
handed to reference tools and back.
"""
from __future__ import annotations

import os

import numpy as np

FOUNDRY_ARRAYS = ("solid", "prim", "node", "tran", "itra", "inst", "plan")
# CSGFoundry::save_ writes plan as (n,1,4) (CSG/CSGFoundry.cc:2769-2800); the engine takes (n,4)
FOUNDRY_SHAPES = {"solid": (3, 4), "prim": (4, 4), "node": (4, 4), "tran": (4, 4), "itra": (4, 4), "inst": (4, 4), "plan": (1, 4)}
FOUNDRY_DTYPES = {"solid": np.int32}
STANDARD_DIR = os.path.join("SSim", "stree", "standard")


def _read_names(path: str) -> list[str]:
    if not os.path.exists(path):
        return []
    with open(path) as f:
        return [line.rstrip("\n") for line in f if line.strip()]


def _write_names(path: str, names) -> None:
    with open(path, "w") as f:
        for n in names:
            f.write(f"{n}\n")


def read_meta(npy_path: str) -> dict:
    """the NP sidecar ``<name>_meta.txt`` of ``<name>.npy`` as a dict of strings (key:value lines)"""
    path = npy_path[:-4] + "_meta.txt" if npy_path.endswith(".npy") else npy_path + "_meta.txt"
    meta = {}
    if os.path.exists(path):
        with open(path) as f:
            for line in f:
                line = line.rstrip("\n")
                if ":" in line:
                    k, v = line.split(":", 1)
                    meta[k] = v
    return meta


def write_meta(npy_path: str, meta: dict) -> None:
    path = npy_path[:-4] + "_meta.txt"
    with open(path, "w") as f:
        for k, v in meta.items():
            f.write(f"{k}:{v}\n")


def _check(name: str, a: np.ndarray) -> np.ndarray:
    tail = FOUNDRY_SHAPES[name]
    if name == "plan" and a.ndim == 2 and a.shape[1:] == (4,):
        a = a.reshape(-1, 1, 4)
    if a.ndim != 1 + len(tail) or tuple(a.shape[1:]) != tail:
        raise ValueError(f"{name}.npy has shape {a.shape}, expected (n,{','.join(map(str, tail))})")
    want = FOUNDRY_DTYPES.get(name)
    if want is not None:
        if a.dtype.itemsize != 4:
            raise ValueError(f"{name}.npy must hold 32-bit words, got {a.dtype}")
        return np.ascontiguousarray(a).view(want)
    if a.dtype.itemsize != 4:
        raise ValueError(f"{name}.npy must hold 32-bit words, got {a.dtype}")
    return np.ascontiguousarray(a).view(np.float32)


def load_foundry(fold: str) -> dict:
    """CSGFoundry::load: the arrays (plan optional) plus meshname/mmlabel/meta"""
    if not os.path.isdir(fold):
        raise FileNotFoundError(f"no CSGFoundry directory at {fold}")
    out = {}
    for k in FOUNDRY_ARRAYS:
        p = os.path.join(fold, f"{k}.npy")
        if os.path.exists(p):
            out[k] = _check(k, np.load(p))
            if k == "plan":
                out[k] = out[k].reshape(-1, 4)
        elif k != "plan":
            raise FileNotFoundError(f"{p} missing")
    out.setdefault("plan", np.zeros((0, 4), dtype=np.float32))
    out["meshname"] = _read_names(os.path.join(fold, "meshname.txt"))
    out["mmlabel"] = _read_names(os.path.join(fold, "mmlabel.txt"))
    meta = os.path.join(fold, "meta.txt")
    out["meta"] = open(meta).read() if os.path.exists(meta) else ""
    return out


def save_foundry(fold: str, arrays: dict, meshname=None, mmlabel=None, meta: str = "") -> None:
    os.makedirs(fold, exist_ok=True)
    for k in FOUNDRY_ARRAYS:
        a = arrays.get(k)
        if a is None:
            if k == "plan":
                continue
            a = np.zeros((0,) + FOUNDRY_SHAPES[k], dtype=FOUNDRY_DTYPES.get(k, np.float32))
        if k == "plan" and len(a) == 0:
            continue
        np.save(os.path.join(fold, f"{k}.npy"), _check(k, np.asarray(a)))
    _write_names(os.path.join(fold, "meshname.txt"), meshname or [])
    _write_names(os.path.join(fold, "mmlabel.txt"), mmlabel or [])
    with open(os.path.join(fold, "meta.txt"), "w") as f:
        f.write(meta)


def load_standard(fold: str, hd_factor: int = 20) -> dict:
    """bnd/optical/icdf of SSim/stree/standard as the physics dict of engine.Engine"""
    bnd_path = os.path.join(fold, "bnd.npy")
    bnd = np.load(bnd_path)
    if bnd.ndim != 5 or bnd.shape[1:3] != (4, 2) or bnd.shape[4] != 4 or bnd.dtype not in (np.float32, np.float64):
        raise ValueError(f"bnd.npy has shape {bnd.shape} {bnd.dtype}, expected float64/32 (num_bnd,4,2,num_wl,4)")
    # sstandard writes double; QBnd narrows a wide array before the texture upload
    # (qudarap/QBnd.cc:75-82, NP::MakeNarrowIfWide)
    bnd = bnd.astype(np.float32)
    meta = read_meta(bnd_path)
    if "domain_low" not in meta or "domain_step" not in meta:
        raise ValueError("bnd_meta.txt must give domain_low and domain_step (the texture needs its domain)")
    optical = np.load(os.path.join(fold, "optical.npy"))
    # sstandard::make_optical writes int32 (num_bnd,4,4) (sysrap/sstandard.h:311-330); one row per
    # texture line, as (num_bnd*4,4) here
    if optical.shape in ((bnd.shape[0], 4, 4), (bnd.shape[0] * 4, 4)) and optical.dtype.itemsize == 4:
        optical = optical.reshape(bnd.shape[0] * 4, 4)
    else:
        raise ValueError(f"optical.npy has shape {optical.shape}, expected ({bnd.shape[0]},4,4) 32-bit")
    phys = {"bnd": np.ascontiguousarray(bnd), "optical": np.ascontiguousarray(optical).view(np.uint32),
            "wl_low": float(meta["domain_low"]), "wl_step": float(meta["domain_step"]), "hd_factor": int(hd_factor),
            "bnd_names": _read_names(os.path.join(fold, "bnd_names.txt"))}
    icdf_path = os.path.join(fold, "icdf.npy")
    if os.path.exists(icdf_path):
        icdf = np.load(icdf_path).astype(np.float32)
        if icdf.ndim == 2:
            icdf = icdf[:, :, None]
        if icdf.ndim != 3 or icdf.shape[1:] != (4096, 1) or icdf.shape[0] not in (1, 3):
            raise ValueError(f"icdf.npy has shape {icdf.shape}, expected (1 or 3, 4096, 1)")
        phys["icdf"] = np.ascontiguousarray(icdf)
    return phys


def save_standard(fold: str, phys: dict, bnd_names=None) -> None:
    os.makedirs(fold, exist_ok=True)
    # the reference's dtypes and shapes: bnd double with its domain metadata, optical int32
    # (num_bnd,4,4), icdf double (sysrap/sstandard.h:311-330, 495-506)
    bnd = np.ascontiguousarray(phys["bnd"], np.float64)
    p = os.path.join(fold, "bnd.npy")
    np.save(p, bnd)
    lo, step = float(phys.get("wl_low", 60.0)), float(phys.get("wl_step", 1.0))
    hi = lo + step * (bnd.shape[3] - 1)
    write_meta(p, {"domain_low": f"{lo:g}", "domain_high": f"{hi:g}", "domain_step": f"{step:g}", "domain_range": f"{hi - lo:g}"})
    opt = np.ascontiguousarray(phys["optical"], np.uint32).view(np.int32)
    np.save(os.path.join(fold, "optical.npy"), opt.reshape(bnd.shape[0], 4, 4))
    icdf = phys.get("icdf")
    if icdf is not None:
        icdf = np.ascontiguousarray(icdf, np.float64)
        np.save(os.path.join(fold, "icdf.npy"), icdf.reshape(icdf.shape[0], icdf.shape[1], 1))
    _write_names(os.path.join(fold, "bnd_names.txt"), bnd_names or phys.get("bnd_names") or [])


def load_geom(cfbase: str, hd_factor: int = 20) -> tuple[dict, dict]:
    """(geometry, physics) from ``<cfbase>/CSGFoundry`` and its ``SSim/stree/standard``
    (``$VAR`` and ``~`` in cfbase are expanded)"""
    fold = os.path.join(os.path.expanduser(os.path.expandvars(cfbase)), "CSGFoundry")
    geom = load_foundry(fold)
    phys = load_standard(os.path.join(fold, STANDARD_DIR), hd_factor)
    return geom, phys


def save_geom(cfbase: str, geom: dict, phys: dict, meshname=None, bnd_names=None) -> None:
    fold = os.path.join(cfbase, "CSGFoundry")
    save_foundry(fold, geom, meshname=meshname)
    save_standard(os.path.join(fold, STANDARD_DIR), phys, bnd_names)
