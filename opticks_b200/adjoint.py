"""Differentiable expected hits per sensor through a hand-written score-function adjoint.

theta (32) = absorption length, Rayleigh length, reemission probability and refractive index of
one material (the liquid scintillator in the detector) in 8 wavelength bins over [wl_lo, wl_hi).
The device pass (phx_adjoint_device) simulates the photons with those properties and returns the
hits per sensor H_s and J[s, k] = sum over hits on s of d log p(path) / d theta_k, an unbiased
estimator of d E[H_s] / d theta_k.  ``ExpectedHits`` wraps that as a torch.autograd.Function:
forward returns H (num_sensor), backward returns grad_H @ J.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib

KINDS = ("absorption_length", "rayleigh_length", "reemission_prob", "rindex")
C_MM_PER_NS = 299.792458


def nominal_theta(phys: dict, mat_line: int, wl_lo: float = 300.0, wl_hi: float = 620.0,
                  wl_low: float = 60.0, wl_step: float = 1.0) -> np.ndarray:
    """theta from a material's current table: the property at each bin centre"""
    bnd = phys["bnd"]
    b, j = divmod(mat_line, 4)
    binw = (wl_hi - wl_lo) / 8.0
    th = np.zeros(32, np.float32)
    for k in range(8):
        lam = wl_lo + (k + 0.5) * binw
        i = int(round((lam - wl_low) / wl_step))
        n, la, ls, w = bnd[b, j, 0, i]
        th[k], th[8 + k], th[16 + k], th[24 + k] = la, ls, w, n
    return th


def retabulate(phys: dict, theta, mat_line: int, wl_lo: float = 300.0, wl_hi: float = 620.0,
               wl_low: float = 60.0, wl_step: float = 1.0) -> dict:
    """the property tables the device pass uses: every omat/imat line of the material of
    mat_line holds theta on its samples in [wl_lo, wl_hi) (group velocity c/n there)"""
    theta = np.asarray(theta, np.float32)
    bnd = np.array(phys["bnd"], dtype=np.float32, copy=True)
    opt = np.asarray(phys["optical"], np.uint32)
    mat = opt[mat_line, 0]
    nb, _, _, nwl, _ = bnd.shape
    lam = (wl_low + wl_step * np.arange(nwl)).astype(np.float32)
    binw = np.float32((wl_hi - wl_lo) / 8.0)
    sel = (lam >= wl_lo) & (lam < wl_hi)
    bins = np.minimum(7, np.floor((lam - np.float32(wl_lo)) / binw).astype(np.int64))
    for b in range(nb):
        for j in (0, 3):
            if opt[4 * b + j, 0] != mat:
                continue
            g0 = bnd[b, j, 0]
            g1 = bnd[b, j, 1]
            g0[sel, 0] = theta[24 + bins[sel]]
            g0[sel, 1] = theta[bins[sel]]
            g0[sel, 2] = theta[8 + bins[sel]]
            g0[sel, 3] = theta[16 + bins[sel]]
            g1[sel, 0] = np.float32(C_MM_PER_NS) / theta[24 + bins[sel]]
    out = dict(phys)
    out["bnd"] = bnd
    return out


PATHWISE = 0x1   # phx_adjoint_device flag: the refracted direction's change with n, carried as a tangent


def adjoint_device(engine, gs_dev, num_photon: int, event: int, theta, mat_line: int, wl_lo: float, wl_hi: float,
                   hits_dev, grad_dev, stream: int = 0, pathwise: bool = True) -> None:
    """one adjoint pass: hits per sensor and their score sums (see phx_adjoint_device); pathwise
    False gives the score terms alone (the rindex rows then hold the Fresnel score only)"""
    th = np.ascontiguousarray(np.asarray(theta, dtype=np.float32).reshape(32))
    G = gs_dev.numel() // 24
    _lib.check(_lib.lib().phx_adjoint_device(engine._h, C.c_void_p(gs_dev.data_ptr()), int(G), int(num_photon), int(event),
                                             th.ctypes.data_as(C.c_void_p), int(mat_line), float(wl_lo), float(wl_hi),
                                             C.c_void_p(hits_dev.data_ptr()), C.c_void_p(grad_dev.data_ptr()),
                                             PATHWISE if pathwise else 0, C.c_void_p(stream) if stream else None),
               "phx_adjoint_device")


def make_function(torch):
    """the autograd.Function class bound to a torch module (imported lazily)"""

    class ExpectedHits(torch.autograd.Function):
        @staticmethod
        def forward(ctx, theta, engine, gs_dev, num_photon, event, mat_line, wl_lo, wl_hi):
            dev = gs_dev.device
            ns = engine.num_sensor
            hits = torch.zeros((ns,), dtype=torch.float64, device=dev)
            grad = torch.zeros((ns, 32), dtype=torch.float64, device=dev)
            adjoint_device(engine, gs_dev, num_photon, event, theta.detach().cpu().numpy(), mat_line, wl_lo, wl_hi,
                           hits, grad, torch.cuda.current_stream(dev).cuda_stream)
            ctx.save_for_backward(grad)
            ctx.theta_dtype = theta.dtype
            ctx.theta_device = theta.device
            return hits

        @staticmethod
        def backward(ctx, grad_hits):
            (J,) = ctx.saved_tensors
            g = (grad_hits.to(J.dtype).reshape(1, -1) @ J).reshape(32)
            return g.to(ctx.theta_device, ctx.theta_dtype), None, None, None, None, None, None, None

    return ExpectedHits


def expected_hits(theta, engine, gs_dev, num_photon: int, event: int = 0, mat_line: int = 11,
                  wl_lo: float = 300.0, wl_hi: float = 620.0):
    import torch
    return make_function(torch).apply(theta, engine, gs_dev, num_photon, event, mat_line, wl_lo, wl_hi)
