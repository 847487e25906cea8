"""The arithmetic of the tet search's candidate filter, checked in float32 on the CPU.

The filter keeps a candidate when, over the critical tets, min min(det, fma(-thr, L^3, det^2))
> 0, with thr = qLast - (|qLast| 2^-14 + 1e-37) lying just below the current ring key qLast > 0
and det, det^2, L^3 = (L L) L the float32 values the key det^2 / L^3 is formed from. Exactness
needs: every tet whose key fl(det^2 / L^3) is at least qLast gives a positive value (so no
candidate that can beat qLast is dropped), and det <= 0 never passes. fma is one rounding of the
exact det^2 - thr L^3, reproduced here in float64 (the 24 x 24-bit product thr L^3 is exact in
float64, and the sign of the difference survives its rounding)."""
import numpy as np


def _f32(x):
    return np.asarray(x, dtype=np.float32)


def _survives(det, L, thr):
    det, L, thr = _f32(det), _f32(L), _f32(thr)
    L3 = _f32(_f32(L * L) * L)
    d2 = _f32(det * det)
    s = _f32(d2.astype(np.float64) - thr.astype(np.float64) * L3.astype(np.float64))
    return np.minimum(det, s) > 0


def _key(det, L):
    det, L = _f32(det), _f32(L)
    L3 = _f32(_f32(L * L) * L)
    return np.where(det < 0, det, _f32(_f32(det * det) / L3))


def _thr(q):
    q = _f32(q)
    return _f32(q - _f32(_f32(np.abs(q) * np.float32(2.0 ** -14)) + np.float32(1e-37)))


def test_every_tet_at_or_above_the_current_key_survives():
    r = np.random.default_rng(0)
    n = 2_000_000
    # scaled local coordinates: ring extents near 1, dets and edge sums of a jittered lattice
    L = _f32(r.uniform(0.05, 12.0, n))
    det = _f32(r.uniform(-0.5, 1.0, n) * np.sqrt(L) ** 3)
    key = _key(det, L)
    # current keys just at, just below and well below each tet's key
    for q in (key, _f32(key * np.float32(1 - 2 ** -20)), _f32(key * np.float32(0.5))):
        pos = q > 0
        ok = _survives(det[pos], L[pos], _thr(q[pos]))
        assert ok.all(), int((~ok).sum())


def test_no_tet_with_det_at_or_below_zero_passes():
    r = np.random.default_rng(1)
    n = 1_000_000
    L = _f32(r.uniform(1e-3, 12.0, n))
    det = _f32(-r.uniform(0.0, 1.0, n) * np.sqrt(L) ** 3)
    thr = _f32(r.uniform(1e-30, 0.2, n))
    assert not _survives(det, L, thr).any()
    assert not _survives(_f32([0.0, -0.0, -1e-30, -3.0]), _f32([1e-3, 1.0, 5.0, 1.0]), _f32([1e-30] * 4)).any()
