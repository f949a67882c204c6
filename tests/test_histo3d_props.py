"""Histogram3D maps on random scanners: properties, and the reference.

The reference checks its bin maps by properties over random scanners
(unit_tests/datastruct/test_Histogram3D.cpp:118-378: bin <-> detector pair
round trip, detector-swap symmetry, uniqueness, coverage), with no golden
vectors.  The same properties are checked here on the oracle for 25 seeded
scanners, and the oracle's maps equal the reference library's bit for bit on
each of them (when the reference is built).  tests/test_gpu_parity.py checks
the device maps against the oracle on the same scanners.  Integer work:
everything is exact.
"""
import numpy as np
import pytest

import pyoracle as po

UINT64_MAX = np.iinfo(np.uint64).max


def random_scanners(n=25, seed=20261203):
    # The reference test's domain (even crystals per ring, minimum angle
    # difference 2 .. detsPerRing/2, any ring difference), sized so that every
    # crystal pair can be enumerated: up to 64 crystals per ring, 8 rings and
    # 3 DOI layers.
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        dpr = 2 * int(rng.integers(2, 33))          # even, 4..64
        rings = int(rng.integers(1, 9))
        doi = int(rng.integers(1, 4))
        mrd = int(rng.integers(0, rings))
        mad = int(rng.integers(2, dpr // 2 + 1))
        out.append(po.Scanner(200.0, 1.0, 1.0, 10.0, 200.0, dpr, rings, doi, mrd,
                              mad, 2))
    return out


SCANNERS = random_scanners()


def all_bins(sc):
    return np.arange(int(np.prod(po.histo3d_dims(sc))), dtype=np.uint64)


@pytest.mark.parametrize("i", range(len(SCANNERS)))
def test_histogram_maps_properties(i):
    sc = SCANNERS[i]
    bins = all_bins(sc)
    d1, d2 = po.histo3d_detpairs(sc, bins)
    # Bins whose two crystals coincide are placeholders (both ids 0).
    valid = ~((d1 == 0) & (d2 == 0))
    assert valid.any()
    b, a1, a2 = bins[valid], d1[valid], d2[valid]
    # Round trip and detector-swap symmetry.
    assert np.array_equal(po.histo3d_bins(sc, a1, a2), b)
    assert np.array_equal(po.histo3d_bins(sc, a2, a1), b)
    # Uniqueness: no unordered detector pair belongs to two bins.
    lo, hi = np.minimum(a1, a2).astype(np.uint64), np.maximum(a1, a2).astype(np.uint64)
    key = lo * np.uint64(sc.num_dets) + hi
    assert len(np.unique(key)) == len(key)
    # Coverage: every pair of distinct crystals either has a bin (and then
    # one of the bins above) or is outside the histogram (ring difference
    # or minimum angle difference).
    n = sc.num_dets
    p1, p2 = np.triu_indices(n, 1)
    pb = po.histo3d_bins(sc, p1.astype(np.uint32), p2.astype(np.uint32))
    inside = pb != UINT64_MAX
    assert int(inside.sum()) == len(b)
    assert np.array_equal(np.sort(pb[inside]), np.sort(b))


@pytest.mark.skipif(not po.ref_available(), reason="reference library not built")
@pytest.mark.parametrize("i", range(len(SCANNERS)))
def test_histogram_maps_match_reference(i):
    sc = SCANNERS[i]
    assert po.histo3d_dims(sc) == po.ref_histo3d_dims(sc)
    bins = all_bins(sc)
    d1, d2 = po.histo3d_detpairs(sc, bins)
    r1, r2 = po.ref_histo3d_detpairs(sc, bins)
    assert np.array_equal(d1, r1) and np.array_equal(d2, r2)
    rng = np.random.default_rng(i)
    q1 = rng.integers(0, sc.num_dets, 20000).astype(np.uint32)
    q2 = rng.integers(0, sc.num_dets, 20000).astype(np.uint32)
    keep = q1 != q2
    q1, q2 = q1[keep], q2[keep]
    assert np.array_equal(po.histo3d_bins(sc, q1, q2), po.ref_histo3d_bins(sc, q1, q2))
