"""Iteration ranges and the file names of per-iteration images.

RangeList mirrors the reference's util::RangeList (include/yrt-pet/utils/
RangeList.hpp, src/utils/RangeList.cpp): a sorted list of closed integer
intervals, parsed from strings like "1-3,5", where overlapping or adjacent
intervals merge ([1,3] and [4,6] become [1,6]).  OSEM uses it to choose the
iterations whose image is saved (OSEM::setSaveIterRanges, OSEM.cpp:651-655,
checked after each iteration at OSEM.cpp:345-348).

iteration_filename follows OSEM::saveForCurrentIteration (OSEM.cpp:813-821):
"_iteration" and the 1-based iteration number, zero-padded to the digits of
the iteration count, inserted before the file's extension (".gz" is kept
with the extension before it, util::addBeforeExtension, src/utils/
Tools.cpp:174-207).
"""
from __future__ import annotations

import math
from typing import List, Tuple


class RangeList:
    def __init__(self, ranges: str = ""):
        self._ranges: List[Tuple[int, int]] = []
        if ranges:
            self.readFromString(ranges)

    def readFromString(self, ranges: str):
        for part in ranges.split(","):
            limits = part.split("-")
            if len(limits) == 1:
                begin = end = int(limits[0])
            elif len(limits) == 2:
                begin, end = int(limits[0]), int(limits[1])
            else:
                raise ValueError(f"Could not parse range {part!r}")
            self.insertSorted(begin, end)

    @staticmethod
    def makeRangeListStep(begin: int, end_incl: int, step: int = 1) -> "RangeList":
        r = RangeList()
        if step == 1:
            r.insertSorted(begin, end_incl)
        else:
            for it in range(begin, end_incl + 1, step):
                r.insertSorted(it, it)
        return r

    def insertSorted(self, begin: int, end: int):
        """Adds [begin, end] and rebuilds the list: intervals sorted by their
        start, overlapping or adjacent ones merged."""
        spans = sorted(self._ranges + [(begin, end)])
        merged: List[List[int]] = []
        for b, e in spans:
            if merged and b <= merged[-1][1] + 1:
                merged[-1][1] = max(merged[-1][1], e)
            else:
                merged.append([b, e])
        self._ranges = [(b, e) for b, e in merged]

    def sort(self):
        ranges, self._ranges = self._ranges, []
        for b, e in ranges:
            self.insertSorted(b, e)

    def get(self) -> List[Tuple[int, int]]:
        return list(self._ranges)

    def getSizeTotal(self) -> int:
        return sum(e - b + 1 for b, e in self._ranges)

    def isIn(self, idx: int) -> bool:
        return any(b <= idx <= e for b, e in self._ranges)

    def contains(self, idx: int) -> bool:
        return self.isIn(idx)

    def empty(self) -> bool:
        return not self._ranges

    def __getitem__(self, i: int) -> Tuple[int, int]:
        return self._ranges[i]

    def __len__(self) -> int:
        return len(self._ranges)

    def __repr__(self) -> str:
        return ", ".join(f"[{b},{e}]" for b, e in self._ranges)


def number_of_digits(n: int) -> int:
    """Decimal digits of n >= 0 (util::numberOfDigits)."""
    return 1 if n == 0 else int(math.ceil(math.log10(n + 1)))


def pad_zeros(number: int, num_digits: int) -> str:
    pad = num_digits - number_of_digits(number)
    if pad < 0:
        raise ValueError("The number given in pad_zeros exceeds the number "
                         "of digits allowed")
    return "0" * pad + str(number)


def extension_start(fname: str) -> int:
    """Index of the extension's dot (a ".gz" suffix stays with the extension
    before it); len(fname) when there is none."""
    pos = len(fname) - 1
    last_two = ["", ""]
    while pos >= 0:
        ch = fname[pos]
        if ch == "." and not (last_two[0] == "g" and last_two[1] == "z"):
            return pos
        last_two[1] = last_two[0]
        last_two[0] = ch
        pos -= 1
    return len(fname)


def add_before_extension(fname: str, addition: str) -> str:
    p = extension_start(fname)
    return fname[:p] + addition + fname[p:]


def iteration_filename(path: str, iteration: int, num_iterations: int) -> str:
    """File name of the image after iteration `iteration` (0-based) of
    num_iterations."""
    return add_before_extension(
        path, "_iteration" + pad_zeros(iteration + 1, number_of_digits(num_iterations)))
