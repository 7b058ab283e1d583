"""TEST INFRASTRUCTURE ONLY — CPU restatement of the reference's hit merge, the checker for
phx_merge_hits.  Never called by the product path.

Follows SPM::merge_partial_select (sysrap/SPM.cu:110-200): select by any-bit flag mask
(sphoton::select_pred, sysrap/sphoton.h:315-319), key (identity << 48) | unsigned(time / window)
(key_functor, sysrap/sphoton.h:292-301 and sysrap/sphotonlite.h:68-77), stable sort by key
(thrust::sort_by_key on integer keys is a stable radix sort), then a left fold of reduce_op over each
run of equal keys (sysrap/sphoton.h:303-313, sysrap/sphotonlite.h:79-91).

Two forms: ``merge_fold`` literally folds reduce_op record by record (pure Python; small inputs) and
``merge`` does the same with numpy group operations; the tests check one against the other.

Division: the reference is compiled with --use_fast_math, numpy divides in IEEE float32.  Both are
exact for power-of-two windows; otherwise a record whose time / window lies within a few ulp of an
integer may fall in a neighbouring bucket.
"""
from __future__ import annotations

import numpy as np

ALREADY_HITMASK_SELECTED = 0xFFFFFFFF
# word offsets: (words per record, time, hitcount word (hi16), identity word, identity mask, flagmask)
LAYOUT = {0: (16, 3, 7, 13, 0xFFFFFF, 15), 1: (4, 1, 0, 0, 0xFFFF, 3)}


def record_kind(rec: np.ndarray) -> int:
    if rec.ndim == 3 and rec.shape[1:] == (4, 4):
        return 0
    if rec.ndim == 2 and rec.shape[1] == 4:
        return 1
    raise ValueError(rec.shape)


def _bucket(t: np.ndarray, tw: float) -> np.ndarray:
    """static_cast<unsigned>(t / tw) as the GPU converts it (round toward zero, NaN -> 0, saturating)"""
    q = (t.astype(np.float32) / np.float32(tw)).astype(np.float64)
    q = np.where(np.isnan(q), 0.0, q)
    return np.clip(np.trunc(q), 0, 2**32 - 1).astype(np.uint64)


def keys(rec: np.ndarray, tw: float) -> np.ndarray:
    W, T, _, I, IM, _ = LAYOUT[record_kind(rec)]
    u = np.ascontiguousarray(rec).view(np.uint32).reshape(len(rec), W)
    ident = (u[:, I] & np.uint32(IM)).astype(np.uint64) & np.uint64(0xFFFF)
    t = u[:, T].view(np.float32)
    return (ident << np.uint64(48)) | _bucket(t, tw)


def select(rec: np.ndarray, mask: int) -> np.ndarray:
    if mask == ALREADY_HITMASK_SELECTED:
        return np.ascontiguousarray(rec)
    W, _, _, _, _, F = LAYOUT[record_kind(rec)]
    u = np.ascontiguousarray(rec).view(np.uint32).reshape(len(rec), W)
    return np.ascontiguousarray(rec[(u[:, F] & np.uint32(mask)) != 0])


def _reduce_op(a: np.ndarray, b: np.ndarray, lite: int) -> np.ndarray:
    """reduce_op(a, b) on single records viewed as uint32 words"""
    W, T, HC, I, IM, F = LAYOUT[lite]
    ta, tb = a[T:T + 1].view(np.float32)[0], b[T:T + 1].view(np.float32)[0]
    tmin = np.float32(np.fmin(ta, tb))
    hc = (int(a[HC] >> 16) + int(b[HC] >> 16)) & 0xFFFF
    if lite:
        r = a.copy()
        r[T:T + 1] = np.array([tmin], np.float32).view(np.uint32)
        r[F] = a[F] | b[F]
        r[0] = np.uint32((hc << 16) | int(a[0] & 0xFFFF))
    else:
        r = (a if tmin == ta else b).copy()
        r[F] = a[F] | b[F]
        r[HC] = np.uint32((int(r[HC]) & 0xFFFF) | (hc << 16))
    return r


def merge_fold(rec: np.ndarray, mask: int = ALREADY_HITMASK_SELECTED, tw: float = 1.0) -> np.ndarray:
    """literal restatement: select, stable sort by key, left fold of reduce_op per key run"""
    lite = record_kind(rec)
    W = LAYOUT[lite][0]
    s = select(rec, mask)
    if len(s) == 0 or tw == 0.0:
        return s
    k = keys(s, tw)
    order = np.argsort(k, kind="stable")
    u = s.view(np.uint32).reshape(len(s), W)
    out = []
    acc = None
    prev = None
    for j in order:
        if prev is not None and k[j] == prev:
            acc = _reduce_op(acc, u[j], lite)
        else:
            if acc is not None:
                out.append(acc)
            acc = u[j].copy()
        prev = k[j]
    out.append(acc)
    return np.stack(out).view(rec.dtype).reshape((len(out),) + rec.shape[1:])


def _order_time(bits: np.ndarray) -> np.ndarray:
    """monotone u32 order of float32 bits, NaN last (fminf ignores NaN)"""
    b = bits.astype(np.uint32)
    nan = (b & np.uint32(0x7FFFFFFF)) > np.uint32(0x7F800000)
    o = np.where(b & np.uint32(0x80000000), ~b, b | np.uint32(0x80000000))
    return np.where(nan, np.uint32(0xFFFFFFFF), o).astype(np.uint32)


def _unorder_time(o: np.ndarray) -> np.ndarray:
    back = np.where(o & np.uint32(0x80000000), o & np.uint32(0x7FFFFFFF), ~o)
    return np.where(o == np.uint32(0xFFFFFFFF), np.uint32(0x7FC00000), back).astype(np.uint32)


def merge(rec: np.ndarray, mask: int = ALREADY_HITMASK_SELECTED, tw: float = 1.0) -> np.ndarray:
    """numpy form of merge_fold (finite times)"""
    lite = record_kind(rec)
    W, T, HC, I, IM, F = LAYOUT[lite]
    s = select(rec, mask)
    if len(s) == 0 or tw == 0.0:
        return s
    k = keys(s, tw)
    u = s.view(np.uint32).reshape(len(s), W)
    pos = np.arange(len(s))
    order = np.argsort(k, kind="stable")
    ks = k[order]
    starts = np.flatnonzero(np.concatenate([[True], ks[1:] != ks[:-1]]))
    fl = np.bitwise_or.reduceat(u[order, F], starts)
    hc = (np.add.reduceat((u[order, HC] >> 16).astype(np.int64), starts) & 0xFFFF).astype(np.uint32)
    tord = _order_time(u[:, T])
    if lite:
        out = u[order[starts]].copy()                      # first record of each run
        out[:, T] = _unorder_time(np.minimum.reduceat(tord[order], starts))
        out[:, 0] = (hc << np.uint32(16)) | (out[:, 0] & np.uint32(0xFFFF))
    else:
        o2 = np.lexsort((pos, tord, k))                   # by key, then time, then input position
        k2 = k[o2]
        st2 = np.flatnonzero(np.concatenate([[True], k2[1:] != k2[:-1]]))
        out = u[o2[st2]].copy()
        out[:, HC] = (out[:, HC] & np.uint32(0xFFFF)) | (hc << np.uint32(16))
    out[:, F] = fl
    return out.view(rec.dtype).reshape((len(out),) + rec.shape[1:])


# ---------------------------------------------------------------- known-answer fixture
EFFICIENCY_COLLECT = 0x1 << 13


def mock_merged(ni: int, tw: float, lite: bool) -> np.ndarray:
    """a merged result with known hit counts: record i has identity = hitcount = 1 + i % 10000 and
    time 100 + 100 f, f = (1 + i % 10000) / 10001, flagmask EC, sorted by key (the fixture of
    qudarap/tests/QEvtTest.cc:482-540 built by sysrap/sutil.h:161-190)"""
    u_dummy = 1 + (np.arange(ni) % 10000)
    f = (u_dummy.astype(np.float32) / np.float32(10001)).astype(np.float32)
    t = (np.float32(100) + f * np.float32(100)).astype(np.float32)
    if lite:
        r = np.zeros((ni, 4), np.uint32)
        r[:, 0] = (u_dummy.astype(np.uint32) << 16) | (u_dummy.astype(np.uint32) & 0xFFFF)
        r[:, 1] = t.view(np.uint32)
        lc = np.clip(np.round(f * 0xFFFF), 0, 0xFFFF).astype(np.uint32)
        r[:, 2] = (lc << 16) | lc
        r[:, 3] = EFFICIENCY_COLLECT
        rec = r.view(np.float32)
    else:
        r = np.zeros((ni, 4, 4), np.float32)
        r[:, 0, 0] = f                                  # payload standing in for the unit-sphere lpos
        r[:, 0, 3] = t
        ru = r.view(np.uint32)
        ru[:, 1, 3] = u_dummy.astype(np.uint32) << 16
        ru[:, 3, 1] = u_dummy.astype(np.uint32)
        ru[:, 3, 3] = EFFICIENCY_COLLECT
        rec = r
    order = np.argsort(keys(rec, tw), kind="stable")
    return np.ascontiguousarray(rec[order])


def unmerge(merged: np.ndarray) -> np.ndarray:
    """each merged record repeated hitcount times with hitcount 1 (sysrap/sutil.h:193-240)"""
    lite = record_kind(merged)
    W, _, HC, _, _, _ = LAYOUT[lite]
    u = merged.view(np.uint32).reshape(len(merged), W)
    hc = (u[:, HC] >> 16).astype(np.int64)
    out = np.repeat(u, hc, axis=0)
    out[:, HC] = (out[:, HC] & np.uint32(0xFFFF)) | np.uint32(1 << 16)
    return out.view(merged.dtype).reshape((len(out),) + merged.shape[1:])
