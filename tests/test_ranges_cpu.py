"""RangeList and the per-iteration file names (OSEM::setSaveIterRanges).

Known answers follow the reference's util::RangeList (src/utils/
RangeList.cpp: sorted, overlapping and adjacent intervals merged) and
OSEM::saveForCurrentIteration (src/recon/OSEM.cpp:813-821 with
util::addBeforeExtension, util::padZeros, util::numberOfDigits).
"""
import pytest

from pyyrtpet_b200.ranges import (RangeList, add_before_extension,
                                  iteration_filename, number_of_digits,
                                  pad_zeros)


def test_parse_merge_and_membership():
    r = RangeList("5,1-3,4,10-12,11")
    assert r.get() == [(1, 5), (10, 12)]
    assert repr(r) == "[1,5], [10,12]"
    assert r.getSizeTotal() == 8
    assert [i for i in range(14) if r.isIn(i)] == [1, 2, 3, 4, 5, 10, 11, 12]
    assert r.contains(11) and not r.contains(9)
    assert r[1] == (10, 12) and len(r) == 2
    assert RangeList().empty() and not r.empty()
    r.insertSorted(7, 8)
    assert r.get() == [(1, 5), (7, 8), (10, 12)]
    r.insertSorted(6, 6)
    assert r.get() == [(1, 8), (10, 12)]


def test_step_ranges():
    assert RangeList.makeRangeListStep(2, 9, 3).get() == [(2, 2), (5, 5), (8, 8)]
    assert RangeList.makeRangeListStep(2, 9, 1).get() == [(2, 9)]
    assert RangeList.makeRangeListStep(1, 4, 2).get() == [(1, 1), (3, 3)]


def test_bad_range_string():
    with pytest.raises(ValueError):
        RangeList("1-2-3")


def test_iteration_file_names():
    assert number_of_digits(0) == 1 and number_of_digits(9) == 1
    assert number_of_digits(10) == 2 and number_of_digits(99) == 2
    assert number_of_digits(100) == 3
    assert pad_zeros(7, 3) == "007"
    with pytest.raises(ValueError):
        pad_zeros(1000, 3)
    assert add_before_extension("img.nii", "_x") == "img_x.nii"
    assert add_before_extension("img.nii.gz", "_x") == "img_x.nii.gz"
    assert add_before_extension("dir.v1/img", "_x") == "dir_x.v1/img"
    assert add_before_extension("img", "_x") == "img_x"
    assert iteration_filename("out/recon.nii.gz", 2, 10) == "out/recon_iteration03.nii.gz"
    assert iteration_filename("recon.npy", 0, 5) == "recon_iteration1.npy"
