"""The serving loop (ft_b200_server_*): requests of different sizes, frame
counts and null-model settings, admitted together, share their stacking
launches; each result must equal the same search run alone (ft_b200_search),
which the search tests pin to the reference's search()."""
import threading

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def _requests():
    g = golden("search_small.npz")
    raw, mjd, exp = g["raw"], g["mjd"], g["exptime"]
    n = raw.shape[0]
    rng = np.random.default_rng(5)
    reqs = [
        (raw, mjd, exp, dict(fwhm_px=2.5, null_runs=2)),
        (raw[:, 8:, 4:].copy(), mjd, exp, dict(fwhm_px=2.5, null_runs=3)),
        (raw[: n - 3], mjd[: n - 3], exp[: n - 3], dict(fwhm_px=0.0, null_runs=1)),
        (raw, mjd, exp, dict(fwhm_px=2.5, threshold_snr=4.5)),
        (raw[:, :, ::-1].copy(), mjd, exp, dict(fwhm_px=2.0, null_runs=2, seed=99)),
        ((raw + rng.normal(0, 3, raw.shape)).astype(np.float32), mjd, exp, dict(fwhm_px=2.5, null_runs=2)),
    ]
    return reqs


def _same(a, b):
    assert a["threshold"] == b["threshold"] and a["method"] == b["method"]
    assert a["fwhm"] == b["fwhm"] and a["n_velocities"] == b["n_velocities"]
    assert np.array_equal(a["null_peaks"], b["null_peaks"])
    assert np.array_equal(a["max_snr"], b["max_snr"], equal_nan=True)
    assert np.array_equal(a["best_v"], b["best_v"])
    assert a["peaks"] == b["peaks"] and a["selected"] == b["selected"]


def test_server_batch_matches_standalone(device):
    import fainttrail_b200 as ftb
    reqs = _requests()
    alone = [device.search(f, m, e, **kw) for f, m, e, kw in reqs]
    srv = ftb.Server(0, 0.0, max_batch=16, workers=1)
    try:
        srv.pause(True)
        tickets = [None] * len(reqs)

        def submit(k):
            f, m, e, kw = reqs[k]
            tickets[k] = srv.submit(f, m, e, **kw)
        th = [threading.Thread(target=submit, args=(k,)) for k in range(len(reqs))]
        for t in th:
            t.start()
        for t in th:
            t.join()
        assert srv.poll(tickets[0], wait_ms=0) is None  # held while paused
        srv.pause(False)
        got = [srv.poll(t) for t in tickets]
        st = srv.stats()
    finally:
        srv.close()
    for a, b in zip(got, alone):
        _same(a, b)
    assert st["completed"] == len(reqs) and st["rounds"] == 1 and st["mean_batch"] == len(reqs)
    assert 0 < st["p50_s"] <= st["p99_s"]


def test_server_two_workers_share_the_queue(device):
    """Two workers' steps in flight on two streams: the held queue is shared
    out, and every result still equals the search run alone."""
    import fainttrail_b200 as ftb
    reqs = _requests()
    alone = [device.search(f, m, e, **kw) for f, m, e, kw in reqs]
    srv = ftb.Server(0, 0.0, max_batch=16, workers=2)
    try:
        srv.pause(True)
        tickets = [srv.submit(f, m, e, **kw) for f, m, e, kw in reqs]
        srv.pause(False)
        got = [srv.poll(t) for t in tickets]
        st = srv.stats()
    finally:
        srv.close()
    for a, b in zip(got, alone):
        _same(a, b)
    assert st["completed"] == len(reqs) and st["rounds"] >= 2


def test_server_streaming_and_errors(device):
    import fainttrail_b200 as ftb
    reqs = _requests()[:3]
    alone = [device.search(f, m, e, **kw) for f, m, e, kw in reqs]
    srv = ftb.Server(0, 0.0, max_batch=2)
    try:
        g = golden("search_small.npz")
        bad = srv.submit(g["raw"][:3], g["mjd"][:3], g["exptime"][:3], fwhm_px=2.5)  # too few frames
        tickets = [srv.submit(f, m, e, **kw) for f, m, e, kw in reqs]
        got = [srv.poll(t) for t in tickets]
        with pytest.raises(RuntimeError, match="frames"):
            srv.poll(bad)
        with pytest.raises(RuntimeError, match="unknown"):
            srv.poll(tickets[0])  # a finished request is handed out once
        st = srv.stats()
    finally:
        srv.close()
    for a, b in zip(got, alone):
        _same(a, b)
    assert st["completed"] == 3 and st["rounds"] >= 2


def test_server_shared_budget_admits_as_memory_frees(device):
    """A budget that holds one request at a time (each needs about 64 MB here):
    the two workers share it, the others wait for memory, and every result still
    equals the search run alone."""
    import fainttrail_b200 as ftb
    reqs = _requests()[:4]
    alone = [device.search(f, m, e, **kw) for f, m, e, kw in reqs]
    srv = ftb.Server(0, 100e6, max_batch=16, workers=2)
    try:
        tickets = [srv.submit(f, m, e, **kw) for f, m, e, kw in reqs]
        got = [srv.poll(t) for t in tickets]
        st = srv.stats()
    finally:
        srv.close()
    for a, b in zip(got, alone):
        _same(a, b)
    assert st["completed"] == len(reqs) and st["rounds"] >= len(reqs)


def test_server_admits_during_a_long_request(device):
    """Continuous batching: a short request submitted while a long one is being
    stacked (thirty null runs, two passes per step) is admitted at the next step
    boundary, its pass shares a launch with the long one's, and it is published
    first; both results equal the searches run alone."""
    import time
    import fainttrail_b200 as ftb
    g = golden("search_small.npz")
    raw, mjd, exp = g["raw"], g["mjd"], g["exptime"]
    long_kw = dict(fwhm_px=2.5, null_runs=30)
    short_kw = dict(fwhm_px=2.5, threshold_snr=4.5)
    short = raw[:, 10:, 10:].copy()
    alone_long = device.search(raw, mjd, exp, **long_kw)
    alone_short = device.search(short, mjd, exp, **short_kw)
    srv = ftb.Server(0, 0.0, max_batch=2, workers=1)
    try:
        t_long = srv.submit(raw, mjd, exp, **long_kw)
        t0 = time.perf_counter()
        while srv.stats()["rounds"] < 1 and time.perf_counter() - t0 < 30:
            time.sleep(0.001)
        t_short = srv.submit(short, mjd, exp, **short_kw)
        got_short = srv.poll(t_short)
        long_pending = srv.poll(t_long, wait_ms=0)
        got_long = long_pending if long_pending is not None else srv.poll(t_long)
        st = srv.stats()
    finally:
        srv.close()
    _same(got_long, alone_long)
    _same(got_short, alone_short)
    assert long_pending is None  # the short request finished while the long one was still stacking
    assert st["completed"] == 2 and st["rounds"] >= 15
