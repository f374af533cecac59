"""Failure paths that fault nothing on the device: a staging wait that runs out
returns an error and leaves the context usable; a search or a served request
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


def test_bounded_staging_wait_reports_and_recovers(backend, oracle):
    """The stacking kernel's staging waits are bounded: with the test knob, every
    staging barrier expects 16 bytes that no copy brings, so each wait gives up
    after about 10 ms of clock, the kernel returns with the error flag set and
    the pass fails with "a device wait timed out"; nothing hangs or faults, and
    the same context then runs the pass normally, bit-identical to the oracle."""
    import ctypes as C
    import numpy as np
    L = ftb.lib()
    L.ft_b200_set_wait_test.argtypes = [C.c_int, C.c_longlong]
    g = golden("stack_nan_table.npz")
    p = ftb.StackPass(g["frames"], t_h=g["t_h"], velocities=g["vel"], min_count=int(g["min_count"]))
    try:
        assert L.ft_b200_set_wait_test(16, 20_000_000) == ftb.FT_B200_OK
        with pytest.raises(RuntimeError, match="timed out"):
            backend.run(p)
    finally:
        assert L.ft_b200_set_wait_test(0, 0) == ftb.FT_B200_OK
    r = backend.run(p)
    dx, dy = oracle.shift_table(g["t_h"], g["vel"])
    ms, bv = oracle.stack(g["frames"], dx, dy, int(g["min_count"]))
    assert np.array_equal(r.max_snr, ms, equal_nan=True) and np.array_equal(r.best_v, bv)
