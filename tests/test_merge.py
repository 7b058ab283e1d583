"""Hit merging oracle (CPU): the numpy form against the literal reduce_op fold, the known-answer
fixture (merge of a shuffled unmerge gives back the merged records), and the per-launch + final
merge equalling one merge of everything."""
import numpy as np
import pytest

from oracle import merge as M

SD = 0x40
EC = M.EFFICIENCY_COLLECT


def random_records(n, lite, rng, num_id=7, tmax=12.0, tq=0.25):
    """records with many (identity, bucket) collisions and exact time ties"""
    ident = rng.integers(0, num_id, n).astype(np.uint32)
    if not lite:
        ident[rng.random(n) < 0.1] |= np.uint32(1 << 17)      # identity bits above 16 drop out of the key
    t = (np.floor(rng.random(n) * tmax / tq) * tq).astype(np.float32)
    hc = rng.integers(1, 4, n).astype(np.uint32)
    fl = rng.choice(np.array([SD, SD | 0x800, 0x8, EC, SD | EC], np.uint32), n)
    if lite:
        r = np.zeros((n, 4), np.uint32)
        r[:, 0] = (hc << 16) | (ident & 0xFFFF)
        r[:, 1] = t.view(np.uint32)
        r[:, 2] = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
        r[:, 3] = fl
        return r.view(np.float32)
    r = rng.normal(size=(n, 4, 4)).astype(np.float32)
    u = r.view(np.uint32)
    r[:, 0, 3] = t
    u[:, 1, 3] = (hc << 16) | rng.integers(0, 2**16, n).astype(np.uint32)
    u[:, 3, 1] = ident
    u[:, 3, 2] = np.arange(n, dtype=np.uint32)
    u[:, 3, 3] = fl
    return r


@pytest.mark.parametrize("lite", [0, 1])
@pytest.mark.parametrize("mask,tw", [(0xFFFFFFFF, 1.0), (SD, 1.0), (SD, 0.5), (EC, 4.0), (SD, 1e9), (SD, 0.0), (0, 1.0)])
def test_numpy_form_equals_fold(lite, mask, tw):
    rng = np.random.default_rng(7 + lite)
    rec = random_records(700, lite, rng)
    a = M.merge_fold(rec, mask, tw)
    b = M.merge(rec, mask, tw)
    assert a.shape == b.shape
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    if tw > 0 and len(a):
        k = M.keys(a, tw)
        assert np.all(k[1:] > k[:-1])


@pytest.mark.parametrize("lite", [0, 1])
def test_known_answer_unmerge_shuffle(lite):
    x = M.mock_merged(3000, 1.0, bool(lite))
    photons = M.unmerge(x)
    W = 4 if lite else 16
    assert len(photons) == int((x.view(np.uint32).reshape(len(x), W)[:, 0 if lite else 7] >> 16).sum())
    photons = photons[np.random.default_rng(42).permutation(len(photons))]
    assert np.array_equal(M.merge(photons, EC, 1.0).view(np.uint32), x.view(np.uint32))
    assert np.array_equal(M.merge_fold(photons[:4000], EC, 1.0).view(np.uint32),
                          M.merge(photons[:4000], EC, 1.0).view(np.uint32))


@pytest.mark.parametrize("lite", [0, 1])
def test_per_launch_then_final_equals_one_merge(lite):
    rng = np.random.default_rng(11)
    rec = random_records(5000, lite, rng, num_id=40, tmax=30.0)
    partial = np.concatenate([M.merge(p, SD, 1.0) for p in np.array_split(rec, 4)])
    final = M.merge(partial, M.ALREADY_HITMASK_SELECTED, 1.0)
    assert np.array_equal(final.view(np.uint32), M.merge(rec, SD, 1.0).view(np.uint32))


def test_empty_and_selection_only():
    rng = np.random.default_rng(3)
    for lite in (0, 1):
        rec = random_records(50, lite, rng)
        assert len(M.merge(rec[:0], SD, 1.0)) == 0
        sel = M.merge(rec, SD, 0.0)
        W = 4 if lite else 16
        fl = rec.view(np.uint32).reshape(50, W)[:, 3 if lite else 15]
        assert np.array_equal(sel.view(np.uint32), rec[(fl & SD) != 0].view(np.uint32))
