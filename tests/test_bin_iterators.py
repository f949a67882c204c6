"""Subset iterators of the path (CPU): the list-mode interleaved subsets and
the Histogram3D phi-interleaved subsets, with the known answers and
properties of the reference's tests (unit_tests/utils/test_BinIterator.cpp:
89-155, BinIterator.cpp:147-198, 261-265).  Integer work: exact."""
import numpy as np
import pytest

import pyyrtpet_b200 as yrt
from pyyrtpet_b200.core import (BinIteratorChronologicalInterleaved,
                                BinIteratorRangeHistogram3D)

SC_ARGS = (64, 4, 4, 10, 300, 256, 16, 1, 15, 2, 1)


def test_chronological_interleaved_known_answers():
    # 13 events in 3 subsets: subset s starts at s, steps by 3 and ends at
    # 12, 10, 11 (test_BinIterator.cpp:115-128).
    for s, end in enumerate((12, 10, 11)):
        it = BinIteratorChronologicalInterleaved(3, 13, s)
        idx = it.indices()
        assert idx[0] == s and it.get(1) == s + 3 and idx[-1] == end
        assert it.size() == len(idx) == len(range(s, 13, 3))


def test_listmode_subsets_partition_the_events():
    # 15000 events in 9 subsets (test_BinIterator.cpp:130-155): the subsets
    # are interleaved iterators whose sizes add up to the event count, and
    # together they visit every event exactly once.
    sc = yrt.Scanner("t", *SC_ARGS)
    lm = yrt.ListModeLUT(sc)
    lm.allocate(15000)
    its = [lm.getBinIter(9, s) for s in range(9)]
    assert all(isinstance(it, BinIteratorChronologicalInterleaved) for it in its)
    assert sum(it.size() for it in its) == 15000
    allidx = np.concatenate([it.indices() for it in its])
    assert np.array_equal(np.sort(allidx), np.arange(15000))
    with pytest.raises(RuntimeError, match="subset index"):
        lm.getBinIter(9, 9)


def test_listmode_subset_size_matches_the_c_abi_range():
    # A subset reaches the C ABI as yrtb_range(start = s, stride = S, count =
    # 0 = "all of the subset"), which the library resolves to
    # ceil((n - s) / S) events: the iterator's size.
    for n in (0, 1, 2, 13, 1000, 1001):
        for S in (1, 3, 7, 10):
            for s in range(S):
                it = BinIteratorChronologicalInterleaved(S, n, s)
                r = it._range()
                avail = 0 if n == 0 or r.start >= n else (n - r.start + r.stride - 1) // r.stride
                assert avail == it.size()


@pytest.mark.parametrize("seed", range(5))
def test_histogram_subsets_partition_the_bins(seed):
    # Random dimensions (test_BinIterator.cpp:186-206): the phi-interleaved
    # subsets visit every bin exactly once, subset s holds the bins with
    # phi = s mod S in (z, phi, r) order, and their sizes add up.
    rng = np.random.default_rng(seed)
    nz, nphi, nr = (int(x) for x in rng.integers(10, 20, 3))
    S = int(rng.integers(1, 6))
    seen = []
    for s in range(S):
        it = BinIteratorRangeHistogram3D(nz, nphi, nr, S, s)
        b = it.indices()
        assert it.size() == len(b)
        phi = (b // nr) % nphi
        assert np.all(phi % S == s)
        assert np.all(np.diff(b) > 0)
        seen.append(b)
    allb = np.concatenate(seen)
    assert np.array_equal(np.sort(allb), np.arange(nz * nphi * nr))


def test_histogram_getbiniter_uses_the_histogram_dims():
    sc = yrt.Scanner("t", *SC_ARGS)
    h = yrt.Histogram3D(sc)
    it = h.getBinIter(12, 5)
    assert isinstance(it, BinIteratorRangeHistogram3D)
    assert (it.numZBin, it.numPhi, it.numR) == (h.numZBin, h.numPhi, h.numR)
    total = sum(h.getBinIter(12, s).size() for s in range(12))
    assert total == h.count()
