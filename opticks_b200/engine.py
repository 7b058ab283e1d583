"""Host-side mirror of the reference's simulate interface over the C ABI.

``Engine`` plays the part of CSGOptiX + QSim (CSGOptiX/CSGOptiX.cc:349 Create, :780
simulate(gs, eventID); qudarap/QSim.cc:436-595): it owns the uploaded geometry, property
textures and RNG states of one device and simulates one event per call.
``CSGOptiXService`` mirrors the python service of CSGOptiX/opticks_CSGOptiX.cc:24-110:
``simulate(gs, eventID)`` takes a (G,6,4) genstep array and returns the (H,4,4) hit array.

Errors raise RuntimeError carrying the library's message (the reference asserts/throws,
qudarap/QUDA_CHECK.h:9-35).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import PhxConfig, PhxGeometry, PhxOutputs, PhxPhysics

# status bits (phx_pod.h)
STATUS_NAMES = {
    0x1: "CSG_STACK", 0x2: "BVH_STACK", 0x4: "LOOP_CAP", 0x8: "HIT_OVERFLOW", 0x10: "RNG_RANGE", 0x20: "QUEUE_WATCHDOG",
    0x40: "INPUT_RANGE",
}

FLAG = dict(CK=0x1, SI=0x2, TO=0x4, AB=0x8, RE=0x10, SC=0x20, SD=0x40, SA=0x80, DR=0x100, SR=0x200, BR=0x400, BT=0x800)
# seqhis nibble (FFS of flag) -> abbreviation, as ana/ and sysrap/OpticksPhoton.hh print them
NIBBLE = {1: "CK", 2: "SI", 3: "TO", 4: "AB", 5: "RE", 6: "SC", 7: "SD", 8: "SA", 9: "DR", 10: "SR", 11: "BR", 12: "BT",
          13: "NA", 14: "EC", 15: "EX"}


def status_names(status: int) -> list[str]:
    return [n for b, n in STATUS_NAMES.items() if status & b]


def seqhis_label(seqhis0: int, seqhis1: int = 0) -> str:
    out = []
    for w in (int(seqhis0), int(seqhis1)):
        for k in range(16):
            nib = (w >> (4 * k)) & 0xF
            if nib == 0:
                return " ".join(out)
            out.append(NIBBLE.get(nib, "??"))
    return " ".join(out)


def mask_from_labels(labels: str) -> int:
    m = 0
    for tok in labels.replace("|", ",").split(","):
        tok = tok.strip()
        if tok:
            m |= FLAG[tok]
    return m


def default_config(**kw) -> PhxConfig:
    cfg = PhxConfig()
    _lib.lib().phx_config_default(C.byref(cfg))
    for k, v in kw.items():
        if not hasattr(cfg, k):
            raise KeyError(k)
        setattr(cfg, k, v)
    return cfg


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def planck_icdf() -> np.ndarray:
    """the black-body wavelength ICDF (4096 float32, nm) torch photons without a wavelength sample"""
    out = np.zeros(4096, np.float32)
    _lib.check(_lib.lib().phx_planck_icdf(_ptr(out), 4096), "phx_planck_icdf")
    return out


class Engine:
    def __init__(self, geometry: dict, physics: dict, config: PhxConfig | dict | None = None, device: int = 0):
        L = _lib.lib()
        g = {k: np.ascontiguousarray(v) for k, v in geometry.items()}
        self._keep = dict(g)
        node = g["node"].astype(np.float32, copy=False)
        prim = g["prim"].astype(np.float32, copy=False)
        solid = g["solid"].astype(np.int32, copy=False)
        inst = g["inst"].astype(np.float32, copy=False)
        itra = g.get("itra", np.zeros((0, 4, 4), np.float32)).astype(np.float32, copy=False)
        plan = g.get("plan", np.zeros((0, 4), np.float32)).astype(np.float32, copy=False)
        self._keep.update(node=node, prim=prim, solid=solid, inst=inst, itra=itra, plan=plan)
        geo = PhxGeometry(_ptr(node), len(node), _ptr(prim), len(prim), _ptr(solid), len(solid),
                          _ptr(inst), len(inst), _ptr(itra), len(itra), _ptr(plan), len(plan))
        bnd = np.ascontiguousarray(physics["bnd"], dtype=np.float32)
        optical = np.ascontiguousarray(physics["optical"], dtype=np.uint32)
        icdf = physics.get("icdf")
        icdf = None if icdf is None else np.ascontiguousarray(icdf, dtype=np.float32)
        self._keep.update(bnd=bnd, optical=optical, icdf=icdf)
        phys = PhxPhysics(_ptr(bnd), bnd.shape[0], bnd.shape[3], float(physics.get("wl_low", 60.0)),
                          float(physics.get("wl_step", 1.0)), _ptr(optical),
                          _ptr(icdf), 0 if icdf is None else icdf.shape[0], 0 if icdf is None else icdf.shape[1],
                          int(physics.get("hd_factor", 20)))
        if config is None:
            config = default_config()
        elif isinstance(config, dict):
            config = default_config(**config)
        self.config = config
        self.num_sensor = int(config.num_sensor)
        h = C.c_void_p()
        _lib.check(L.phx_create(C.byref(geo), C.byref(phys), C.byref(config), int(device), C.byref(h)), "phx_create")
        self._h = h
        self.device = device

    # ------------------------------------------------------------------ lifecycle
    def close(self) -> None:
        if getattr(self, "_h", None):
            _lib.lib().phx_destroy(self._h)
            self._h = None

    LAUNCH_FIELDS = ("kernel_mode", "block", "regroup", "chunk", "use_graph", "wave_pool", "wave_refill", "wave_rounds",
                     "wave_tail", "adj_wave_rounds")

    def set_launch_config(self, **kw) -> None:
        """change the launch shape of later calls (fields of LAUNCH_FIELDS); results do not change"""
        for k, v in kw.items():
            if k not in self.LAUNCH_FIELDS:
                raise KeyError(f"{k} is not a launch field")
            setattr(self.config, k, v)
        _lib.check(_lib.lib().phx_set_launch_config(self._h, C.byref(self.config)), "phx_set_launch_config")

    def trim(self) -> int:
        """release the device memory grown for calls (wavefront pool and the like); returns bytes freed"""
        b = C.c_int64(0)
        _lib.check(_lib.lib().phx_trim(self._h, C.byref(b)), "phx_trim")
        return int(b.value)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ------------------------------------------------------------------ simulate
    def simulate(self, gs: np.ndarray, eventID: int = 0, photon: bool = True, seq: bool = True, hit: bool = True,
                 sensor_hits: bool = False) -> dict:
        """One event from host gensteps; returns numpy photon (N,4,4), seq (N,2,2) u64, hit (H,4,4)."""
        gs = np.ascontiguousarray(gs, dtype=np.float32).reshape(-1, 6, 4)
        n = int(_lib.lib().phx_count_photons(_ptr(gs), len(gs)))
        ph = np.empty((n, 4, 4), np.float32) if photon else None
        sq = np.empty((n, 2, 2), np.uint64) if seq else None
        ht = np.empty((n, 4, 4), np.float32) if hit else None
        sh = np.empty((self.num_sensor,), np.uint32) if (sensor_hits and self.num_sensor > 0) else None
        out = PhxOutputs(_ptr(ph), _ptr(sq), _ptr(ht), n if hit else 0, _ptr(sh), 0, 0, 0)
        _lib.check(_lib.lib().phx_simulate(self._h, _ptr(gs), len(gs), int(eventID), C.byref(out)), "phx_simulate")
        res = {"num_photon": int(out.num_photon), "num_hit": int(out.num_hit), "status": int(out.status)}
        if ph is not None:
            res["photon"] = ph
        if sq is not None:
            res["seq"] = sq
        if ht is not None:
            res["hit"] = ht[: int(out.num_hit)]
        if sh is not None:
            res["sensor_hits"] = sh
        return res

    def simulate_into(self, gs: np.ndarray, eventID: int, photon: np.ndarray | None, seq: np.ndarray | None,
                      hit: np.ndarray | None, sensor_hits: np.ndarray | None = None) -> dict:
        """Host API into caller-owned (e.g. pinned) arrays sized for the event's photon count."""
        out = PhxOutputs(_ptr(photon), _ptr(seq), _ptr(hit), 0 if hit is None else len(hit), _ptr(sensor_hits), 0, 0, 0)
        _lib.check(_lib.lib().phx_simulate(self._h, _ptr(gs), len(gs), int(eventID), C.byref(out)), "phx_simulate")
        return {"num_photon": int(out.num_photon), "num_hit": int(out.num_hit), "status": int(out.status)}

    def simulate_device(self, gs_dev, num_photon: int, eventID: int = 0, photon=None, seq=None, hit=None,
                        hit_capacity: int = 0, sensor_hits=None, stream: int = 0, photon_offset: int = 0) -> tuple[int, int]:
        """Device path: arguments are torch CUDA tensors (or raw device pointers as ints).
        Returns (num_hit, status)."""
        def dp(t):
            if t is None:
                return None
            return C.c_void_p(t if isinstance(t, int) else t.data_ptr())
        out = PhxOutputs(dp(photon), dp(seq), dp(hit), int(hit_capacity), dp(sensor_hits), 0, 0, 0)
        G = (gs_dev.numel() // 24) if hasattr(gs_dev, "numel") else None
        _lib.check(_lib.lib().phx_simulate_device(self._h, dp(gs_dev), int(G), int(num_photon), int(eventID),
                                                  int(photon_offset), C.byref(out), C.c_void_p(stream) if stream else None),
                   "phx_simulate_device")
        return int(out.num_hit), int(out.status)

    def simulate_batched_device(self, gs_dev, gs_event_dev, num_photon: int, photon=None, seq=None, hit=None,
                                hit_capacity: int = 0, sensor_hits=None, block: int = 0, chunk: int = 0, regroup: int = 0,
                                num_event: int = 0, event_done_ns=None, stream: int = 0) -> tuple[int, int]:
        """Many events in one persistent launch (torch CUDA tensors).  gs_event_dev: int32 event index
        per genstep, non-decreasing.  event_done_ns: optional int64 tensor (num_event+1) receiving the
        device clock when each event finished and, last, when the launch started.  Returns (num_hit, status)."""
        def dp(t):
            return None if t is None else C.c_void_p(t.data_ptr())
        out = PhxOutputs(dp(photon), dp(seq), dp(hit), int(hit_capacity), dp(sensor_hits), 0, 0, 0)
        G = gs_dev.numel() // 24
        _lib.check(_lib.lib().phx_simulate_batched_device(self._h, dp(gs_dev), dp(gs_event_dev), int(G), int(num_photon),
                                                          int(block), int(chunk), int(regroup), int(num_event),
                                                          dp(event_done_ns), C.byref(out),
                                                          C.c_void_p(stream) if stream else None),
                   "phx_simulate_batched_device")
        return int(out.num_hit), int(out.status)

    # ------------------------------------------------------------------ scan / rng
    def scan(self, prim: int, rays: np.ndarray, t_min: float = 0.0) -> np.ndarray:
        rays = np.ascontiguousarray(rays, dtype=np.float32)
        assert rays.ndim == 2 and rays.shape[0] == 6
        n = rays.shape[1]
        out = np.empty((n, 4), np.float32)
        _lib.check(_lib.lib().phx_csg_scan(self._h, int(prim), float(t_min), _ptr(rays), n, _ptr(out)), "phx_csg_scan")
        return out

    def scan_device(self, prim: int, rays_dev, n: int, isect_dev, t_min: float = 0.0, polish: int = 0, stream: int = 0) -> None:
        _lib.check(_lib.lib().phx_csg_scan_device(self._h, int(prim), float(t_min), C.c_void_p(rays_dev.data_ptr()), int(n),
                                                  C.c_void_p(isect_dev.data_ptr()), int(polish),
                                                  C.c_void_p(stream) if stream else None), "phx_csg_scan_device")

    def trace(self, rays: np.ndarray, t_min: float = 0.0, t_max: float = 1e6) -> tuple[np.ndarray, int]:
        """closest hit of each ray (SoA (6,n)) over the whole geometry: (n,2,4) quad2 PRD rows
        (normal, t; lposcost, 0, iindex<<16|identity, globalPrimIdx<<16|boundary) and the status bits"""
        rays = np.ascontiguousarray(rays, dtype=np.float32)
        assert rays.ndim == 2 and rays.shape[0] == 6
        n = rays.shape[1]
        out = np.empty((n, 2, 4), np.float32)
        st = C.c_uint32(0)
        _lib.check(_lib.lib().phx_trace(self._h, _ptr(rays), n, float(t_min), float(t_max), _ptr(out), C.byref(st)), "phx_trace")
        return out, int(st.value)

    def rng_sequence(self, eventID: int, photon_offset: int, num_photon: int, num_per_photon: int) -> np.ndarray:
        out = np.empty((num_photon, num_per_photon), np.float32)
        _lib.check(_lib.lib().phx_rng_sequence(self._h, int(eventID), int(photon_offset), int(num_photon),
                                               int(num_per_photon), _ptr(out)), "phx_rng_sequence")
        return out

    def set_input_photon(self, photon) -> None:
        """SEvt::setInputPhoton: (N,4,4) float32 sphoton rows that INPUT_PHOTON gensteps (gencode 19)
        copy; a torch tensor on the engine's device is used in place (kept alive here), anything
        else is copied to the device; None clears"""
        if photon is None:
            self._input = None
            _lib.check(_lib.lib().phx_set_input_photon(self._h, None, 0), "phx_set_input_photon")
            return
        if hasattr(photon, "data_ptr") and getattr(photon, "is_cuda", False):
            assert photon.dtype.itemsize == 4 and photon.is_contiguous() and photon.shape[1:] == (4, 4)
            self._input = photon
            _lib.check(_lib.lib().phx_set_input_photon_device(self._h, C.c_void_p(photon.data_ptr()), int(photon.shape[0])),
                       "phx_set_input_photon_device")
            return
        a = np.ascontiguousarray(photon, dtype=np.float32).reshape(-1, 4, 4)
        self._input = None
        _lib.check(_lib.lib().phx_set_input_photon(self._h, _ptr(a), len(a)), "phx_set_input_photon")

    def last_call_stats(self) -> dict:
        """kernel launches and wavefront rounds of the last simulate call"""
        k, r, g = C.c_int64(0), C.c_int64(0), C.c_int32(0)
        _lib.check(_lib.lib().phx_last_call_stats(self._h, C.byref(k), C.byref(r), C.byref(g)), "phx_last_call_stats")
        return {"kernel_launches": int(k.value), "wave_rounds": int(r.value), "graph": bool(g.value)}

    # ------------------------------------------------------------------ hit merging
    def merge_hits(self, records: np.ndarray, select_flagmask: int = 0xFFFFFFFF, time_window: float = 1.0) -> np.ndarray:
        """SPM::merge_partial_select on host arrays: sphoton (n,4,4) or sphotonlite (n,4) records in,
        merged records out (ascending (identity, time bucket) key)."""
        rec = np.ascontiguousarray(records)
        lite = _record_kind(rec)
        n = rec.shape[0]
        out = np.empty_like(rec)
        no = C.c_int64(0)
        _lib.check(_lib.lib().phx_merge_hits(self._h, _ptr(rec), int(n), lite, C.c_uint32(select_flagmask & 0xFFFFFFFF),
                                             float(time_window), _ptr(out), int(n), C.byref(no)), "phx_merge_hits")
        return out[: no.value]

    def merge_hits_device(self, records_dev, out_dev, select_flagmask: int = 0xFFFFFFFF, time_window: float = 1.0,
                          stream: int = 0) -> int:
        """device form on torch CUDA tensors of sphoton (n,4,4) or sphotonlite (n,4) 32-bit words;
        out_dev needs as many rows as records_dev.  Returns the number of merged records."""
        shape = tuple(records_dev.shape)
        lite = 1 if (len(shape) == 2 and shape[1] == 4) else 0
        if not lite and shape[1:] != (4, 4):
            raise ValueError(f"records must be (n,4,4) sphoton or (n,4) sphotonlite, got {shape}")
        if tuple(out_dev.shape[1:]) != shape[1:] or out_dev.shape[0] < shape[0]:
            raise ValueError("out_dev must match the record layout and hold as many rows as records_dev")
        no = C.c_int64(0)
        _lib.check(_lib.lib().phx_merge_hits_device(self._h, C.c_void_p(records_dev.data_ptr()), int(shape[0]), lite,
                                                    C.c_uint32(select_flagmask & 0xFFFFFFFF), float(time_window),
                                                    C.c_void_p(out_dev.data_ptr()), int(out_dev.shape[0]), C.byref(no),
                                                    C.c_void_p(stream) if stream else None), "phx_merge_hits_device")
        return int(no.value)


def _record_kind(rec: np.ndarray) -> int:
    if rec.dtype.itemsize != 4:
        raise ValueError("records must be 32-bit words (float32/uint32)")
    if rec.ndim == 3 and rec.shape[1:] == (4, 4):
        return 0
    if rec.ndim == 2 and rec.shape[1] == 4:
        return 1
    raise ValueError(f"records must be (n,4,4) sphoton or (n,4) sphotonlite, got {rec.shape}")


class CSGOptiXService:
    """gensteps in, hits out (CSGOptiX/CSGOptiXService.h, CSGOptiX/opticks_CSGOptiX.cc:24-110)"""

    def __init__(self, geometry: dict, physics: dict, config=None, device: int = 0):
        self.engine = Engine(geometry, physics, config, device)

    def simulate(self, gs: np.ndarray, eventID: int = 0) -> np.ndarray:
        return self.engine.simulate(gs, eventID, photon=False, seq=False, hit=True)["hit"]

    def __repr__(self) -> str:
        return f"CSGOptiXService(device={self.engine.device})"
