"""Host-side checks of the OperatorProjectorDevice mirror (no GPU needed):
the arguments it cannot honour raise instead of being dropped."""
import pytest

import pyyrtpet_b200 as yrt


def test_create_rejects_constraints_and_memory_budget():
    sc = yrt.Scanner("s", 20, 4, 4, 10, 150, 64, 5, 1, 4, 2, 1)
    pp = yrt.ProjectorParams(sc)
    h = yrt.Histogram3D(sc)
    it = h.getBinIter(1, 0)
    op = yrt.OperatorProjectorDevice.create(pp, it)
    assert op.getBinIter() is it
    with pytest.raises(RuntimeError, match="constraints"):
        yrt.OperatorProjectorDevice.create(pp, it, constraints=[object()])
    with pytest.raises(RuntimeError, match="mem_available"):
        yrt.OperatorProjectorDevice.create(pp, it, mem_available=1 << 30)


def test_projection_list_requires_allocation():
    sc = yrt.Scanner("s", 20, 4, 4, 10, 150, 64, 5, 1, 4, 2, 1)
    pl = yrt.ProjectionListOwned(yrt.Histogram3D(sc))
    with pytest.raises(RuntimeError, match="not allocated"):
        pl.getProjectionValue(0)
