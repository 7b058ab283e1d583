"""comparison helpers shared by the GPU parity tests"""
import numpy as np


def seq_match(a, b):
    """fraction of photons with identical seqhis (both words)"""
    return float(np.mean(np.all(a[:, 0, :] == b[:, 0, :], axis=1)))


def close_mask(a, b, rtol=1e-4):
    """per-photon: position, time, direction and polarisation within rtol (relative to the
    position scale, the time, and unit vectors respectively)"""
    scale = np.maximum(np.abs(b[:, 0, :3]).max(1), 1.0)
    pos = np.abs(a[:, 0, :3] - b[:, 0, :3]).max(1) <= rtol * scale
    tim = np.abs(a[:, 0, 3] - b[:, 0, 3]) <= rtol * np.maximum(np.abs(b[:, 0, 3]), 1.0)
    mom = np.abs(a[:, 1, :3] - b[:, 1, :3]).max(1) <= rtol
    pol = np.abs(a[:, 2, :3] - b[:, 2, :3]).max(1) <= rtol
    return pos, tim, mom, pol


def frac_close(a, b, sel, rtol=1e-4):
    """fraction of selected photons whose pos, time, mom, pol all agree within rtol"""
    if not sel.any():
        return 1.0
    pos, tim, mom, pol = close_mask(a[sel], b[sel], rtol)
    return float(np.mean(pos & tim & mom & pol))


def describe(a, b, sel, rtol=1e-4):
    pos, tim, mom, pol = close_mask(a[sel], b[sel], rtol)
    return f"pos {pos.mean():.6f} time {tim.mean():.6f} mom {mom.mean():.6f} pol {pol.mean():.6f}"
