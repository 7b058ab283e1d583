"""Boundary property tables in the layout the reference uploads as textures.

* ``bnd``     (num_bnd, 4, 2, num_wl, 4) float32 : species omat/osur/isur/imat, two float4 groups,
  wavelength samples on the 60..820 nm 1 nm domain (sysrap/sdomain.h:26-31, qudarap/QBnd.cc:130-165).
  Material group 0 = (rindex, absorption_length, scattering_length, reemission_prob),
  group 1 = (group_velocity, 0, 0, 0); surface group 0 = (detect, absorb, reflect_specular,
  reflect_diffuse) (qudarap/qsim.h:1614-1680).
* ``optical`` (num_bnd*4, 4) uint32 : material lines (index+1, 0, 0, 0); surface lines
  (index+1 or 0, ems, 0, 0) with ems from sysrap/smatsur.h (sysrap/sstandard.h:311-420).
* ``icdf``    (3, 4096, 1) float32 : scintillation wavelength inverse CDF, full range plus the
  two 20x high-definition tails (qudarap/qscint.h:251-258, hd_factor 20).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

WL_LOW, WL_HIGH, WL_STEP = 60.0, 820.0, 1.0
NUM_WL = 761
C_MM_PER_NS = 299.792458

EMS_MATERIAL, EMS_NOSURFACE, EMS_SURFACE, EMS_SENSOR_A = 0, 1, 2, 3


def wavelengths() -> np.ndarray:
    return WL_LOW + WL_STEP * np.arange(NUM_WL, dtype=np.float64)


def _as_curve(v, wl):
    if callable(v):
        return np.asarray(v(wl), dtype=np.float64)
    return np.full_like(wl, float(v))


@dataclass
class Material:
    name: str
    rindex: object = 1.0            # scalar or f(wl_nm)
    absorption_length: object = 1e9  # mm
    scattering_length: object = 1e9  # mm
    reemission_prob: object = 0.0

    def table(self) -> np.ndarray:
        wl = wavelengths()
        n = _as_curve(self.rindex, wl)
        t = np.zeros((2, NUM_WL, 4), dtype=np.float64)
        t[0, :, 0] = n
        t[0, :, 1] = _as_curve(self.absorption_length, wl)
        t[0, :, 2] = _as_curve(self.scattering_length, wl)
        t[0, :, 3] = _as_curve(self.reemission_prob, wl)
        # group velocity c / (n - lambda dn/dlambda)
        dn = np.gradient(n, wl)
        ng = n - wl * dn
        t[1, :, 0] = C_MM_PER_NS / np.clip(ng, 1.0, None)
        return t


@dataclass
class Surface:
    name: str
    detect: float = 0.0
    absorb: float = 1.0
    reflect_specular: float = 0.0
    reflect_diffuse: float = 0.0
    ems: int = EMS_SURFACE

    def table(self) -> np.ndarray:
        t = np.zeros((2, NUM_WL, 4), dtype=np.float64)
        t[0, :, :] = (self.detect, self.absorb, self.reflect_specular, self.reflect_diffuse)
        return t


@dataclass
class BoundaryLib:
    materials: list = field(default_factory=list)
    surfaces: list = field(default_factory=list)
    boundaries: list = field(default_factory=list)   # (omat, osur, isur, imat) names, "" for no surface

    def mat(self, m: Material) -> Material:
        if m.name not in [x.name for x in self.materials]:
            self.materials.append(m)
        return m

    def sur(self, s: Surface) -> Surface:
        if s.name not in [x.name for x in self.surfaces]:
            self.surfaces.append(s)
        return s

    def add(self, omat: str, osur: str, isur: str, imat: str) -> int:
        spec = (omat, osur, isur, imat)
        if spec in self.boundaries:
            return self.boundaries.index(spec)
        self.boundaries.append(spec)
        return len(self.boundaries) - 1

    def material_line(self, name: str) -> int:
        """texture line of a material (4*boundary + OMAT/IMAT) as used for genstep matline"""
        for b, (om, _, _, im) in enumerate(self.boundaries):
            if im == name:
                return 4 * b + 3
            if om == name:
                return 4 * b + 0
        raise KeyError(name)

    def arrays(self) -> dict:
        mi = {m.name: i for i, m in enumerate(self.materials)}
        si = {s.name: i for i, s in enumerate(self.surfaces)}
        mt = {m.name: m.table() for m in self.materials}
        st = {s.name: s.table() for s in self.surfaces}
        nb = len(self.boundaries)
        bnd = np.zeros((nb, 4, 2, NUM_WL, 4), dtype=np.float32)
        optical = np.zeros((nb * 4, 4), dtype=np.uint32)
        for b, (om, os_, is_, im) in enumerate(self.boundaries):
            bnd[b, 0] = mt[om]
            bnd[b, 3] = mt[im]
            optical[4 * b + 0] = (mi[om] + 1, 0, 0, 0)
            optical[4 * b + 3] = (mi[im] + 1, 0, 0, 0)
            for j, sname in ((1, os_), (2, is_)):
                if sname:
                    bnd[b, j] = st[sname]
                    optical[4 * b + j] = (si[sname] + 1, self.surfaces[si[sname]].ems, 0, 0)
                else:
                    optical[4 * b + j] = (0, EMS_NOSURFACE, 0, 0)
        return {"bnd": bnd, "optical": optical}


def icdf_from_pdf(wl: np.ndarray, pdf: np.ndarray, width: int = 4096) -> np.ndarray:
    """(3,width,1) inverse CDF: layer 0 u in [0,1], layer 1 u in [0,0.05], layer 2 u in [0.95,1],
    sampled at texel centres so that the hardware linear lookup at u returns F^-1(u)"""
    cdf = np.concatenate([[0.0], np.cumsum(0.5 * (pdf[1:] + pdf[:-1]) * np.diff(wl))])
    cdf /= cdf[-1]
    keep = np.concatenate([[True], np.diff(cdf) > 0])
    cdf_k, wl_k = cdf[keep], wl[keep]
    x = (np.arange(width, dtype=np.float64) + 0.5) / width
    layers = [x, 0.05 * x, 0.95 + 0.05 * x]
    out = np.stack([np.interp(u, cdf_k, wl_k) for u in layers])
    return out.reshape(3, width, 1).astype(np.float32)


def gaussian_icdf(mu: float = 430.0, sigma: float = 20.0, width: int = 4096) -> np.ndarray:
    wl = np.linspace(mu - 8 * sigma, mu + 8 * sigma, 20001)
    pdf = np.exp(-0.5 * ((wl - mu) / sigma) ** 2)
    return icdf_from_pdf(wl, pdf, width)
