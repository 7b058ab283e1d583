"""The reference's own qsim/CSG path compiled for the CPU (oracle/_ref/libref_cpu_sim.so, the
bench's CPU baseline) against the C restatement on the same detector sample: they draw different
random numbers (the reference's CPU generator against numpy), so the check is statistical: the hit
fraction and the frequencies of the leading seqhis histories agree within their sampling errors."""
import collections

import numpy as np
import pytest

from oracle import oracle as O
from opticks_b200 import scenes

pytestmark = pytest.mark.skipif(not O.have_ref_cpu_sim(), reason="reference CPU build absent")


def _labels(seq):
    from opticks_b200 import engine as E
    return collections.Counter(E.seqhis_label(int(a[0, 0]), int(a[0, 1])) for a in seq)


def test_reference_cpu_path_agrees_with_restatement_in_distribution():
    fd, lib, icdf = scenes.detector()
    phys = lib.arrays()
    phys["icdf"] = icdf
    gs = scenes.detector_gensteps(400, 10000, seed=3, lib=lib)
    gs.view(np.int32)[:, 0, 3] = 10                       # 10 photons from each of 400 vertices
    ph, sq, secs, nt = O.ref_simulate_cpu(fd.arrays(), phys, gs)
    n = len(ph)
    S = O.Scene(fd.arrays(), phys)
    u = np.random.default_rng(5).random((n, 512), dtype=np.float32)
    ph2, sq2, err = S.simulate(gs, u, 0)
    assert err & 1 == 0
    h1 = ((ph.view(np.uint32)[:, 3, 3] & 0x40) != 0).mean()
    h2 = ((ph2.view(np.uint32)[:, 3, 3] & 0x40) != 0).mean()
    se = np.sqrt(h1 * (1 - h1) / n + h2 * (1 - h2) / n)
    print(f"{n} photons, {nt} threads, {n / secs:.0f} photons/s; hit fraction reference CPU {h1:.4f} restatement {h2:.4f}")
    assert abs(h1 - h2) < 4 * se
    a, b = _labels(sq), _labels(sq2)
    for lab, _ in b.most_common(5):
        p1, p2 = a[lab] / n, b[lab] / n
        s = np.sqrt(p1 * (1 - p1) / n + p2 * (1 - p2) / n) + 1e-12
        print(f"   {lab:24s} {p1:.4f} {p2:.4f}")
        assert abs(p1 - p2) < 4 * s, lab
