"""Host logic of the CCD step bound (no GPU): a query status with
IPCB_STATUS_STACK or IPCB_STATUS_ROOT_ITERS refuses the step and counts the
refusal; other bits (the contact BSR's row overflow) do not touch it."""
import pytest

from ipc_warp_b200.contact import QUERY_FAILED, ContactSolverBase


def _bare():
    s = object.__new__(ContactSolverBase)
    s.query_status = 0
    s.ccd_refusals = 0
    return s


@pytest.mark.parametrize("toi,status,bound", [(0.5, 0, 0.45), (1.0, 0, 1.0), (0.5, 1, 0.0), (1.0, 2, 0.0),
                                              (0.25, 3, 0.0), (1.0, 4, 1.0), (0.5, 8, 0.45)])
def test_bound_from_status(toi, status, bound):
    s = _bare()
    assert s._bound_from(toi, status) == pytest.approx(bound)
    assert s.query_status == status
    assert s.ccd_refusals == (1 if status & QUERY_FAILED else 0)


def test_refusals_accumulate():
    s = _bare()
    for st in (1, 0, 2, 0):
        s._bound_from(0.3, st)
    assert s.ccd_refusals == 2 and s.query_status == 0
