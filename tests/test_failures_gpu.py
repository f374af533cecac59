"""Failure paths that fault nothing on the device: a search or a served request
that does not fit the context's HBM budget is refused with an error before any
copy or kernel is queued, and the memory it had charged is released (a second
attempt fails in the same way). The budget check is a host-side count; no
allocation beyond the budget is attempted."""
import pytest

import fainttrail_b200 as ftb
from conftest import golden

pytestmark = pytest.mark.gpu


def test_search_beyond_the_budget_is_refused():
    g = golden("search_small.npz")
    small = ftb.Device(0, 1.0e6)  # the 12 x 80 x 96 search needs several MB
    try:
        errors = []
        for _ in range(2):
            with pytest.raises(RuntimeError, match="HBM budget exceeded") as e:
                small.search(g["raw"], g["mjd"], g["exptime"], fwhm_px=2.5, null_runs=2)
            errors.append(str(e.value))
        assert errors[0] == errors[1]
    finally:
        small.close()


def test_served_request_beyond_the_budget_is_refused():
    g = golden("search_small.npz")
    srv = ftb.Server(0, 1.0e6, max_batch=4, workers=1)
    try:
        ticket = srv.submit(g["raw"], g["mjd"], g["exptime"], fwhm_px=2.5, null_runs=2)
        with pytest.raises(RuntimeError, match="HBM budget exceeded"):
            srv.poll(ticket)
    finally:
        srv.close()
