"""comparison helpers shared by the GPU parity tests"""
import numpy as np


def seq_match(a, b):
    """fraction of photons with identical seqhis (both words)"""
    return float(np.mean(np.all(a[:, 0, :] == b[:, 0, :], axis=1)))


def photon_close(a, b, sel, rtol=1e-4, atol_mm=1e-2):
    """max relative deviation of pos/time/mom/pol over the selected photons"""
    if not sel.any():
        return 0.0
    pa, pb = a[sel], b[sel]
    scale = np.maximum(np.abs(pb[:, 0, :3]).max(1, keepdims=True), 1.0)
    dpos = (np.abs(pa[:, 0, :3] - pb[:, 0, :3]) / scale).max()
    dt = (np.abs(pa[:, 0, 3] - pb[:, 0, 3]) / np.maximum(np.abs(pb[:, 0, 3]), 1e-3)).max()
    dmom = np.abs(pa[:, 1, :3] - pb[:, 1, :3]).max()
    dpol = np.abs(pa[:, 2, :3] - pb[:, 2, :3]).max()
    return float(max(dpos, dt, dmom, dpol))


def frac_close(a, b, sel, rtol=1e-4):
    """fraction of selected photons whose pos, time, mom, pol agree within rtol"""
    pa, pb = a[sel], b[sel]
    if len(pa) == 0:
        return 1.0
    scale = np.maximum(np.abs(pb[:, 0, :3]).max(1), 1.0)
    ok = (np.abs(pa[:, 0, :3] - pb[:, 0, :3]).max(1) <= rtol * scale)
    ok &= np.abs(pa[:, 0, 3] - pb[:, 0, 3]) <= rtol * np.maximum(np.abs(pb[:, 0, 3]), 1.0)
    ok &= np.abs(pa[:, 1, :3] - pb[:, 1, :3]).max(1) <= 10 * rtol
    ok &= np.abs(pa[:, 2, :3] - pb[:, 2, :3]).max(1) <= 10 * rtol
    return float(ok.mean())
