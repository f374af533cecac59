"""Host helpers of the benchmark: the serving stream's motion count (which
decides the per-request work cap) equals the reference velocity grid's size,
the stream is reproducible and within its bounds, and the bench reads the
profiled DRAM traffic of the stack kernel."""
import os
import sys

import numpy as np
import pytest

from fainttrail_b200 import synthetic

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("span_h,vmin,vmax,tol", [(0.325, 6.0, 120.0, 0.125), (0.483, 12.0, 66.0, 0.125),
                                                  (0.2, 0.0, 40.0, 0.5), (1.0, 30.0, 31.0, 0.05)])
def test_motion_count_equals_velocity_grid(oracle, span_h, vmin, vmax, tol):
    grid, _ = oracle.velocity_grid(span_h, vmin, vmax, tol)
    assert synthetic.motion_count(span_h, vmin, vmax, tol) == grid.shape[0]


def test_serving_stream_is_seeded_and_bounded():
    a, da = synthetic.serving_requests(count=12, seed=5)
    b, db = synthetic.serving_requests(count=12, seed=5)
    assert da == db >= 12
    assert [(t, w.width, w.height, w.nframes, w.rate_px_min, w.null_runs) for t, w in a] == \
           [(t, w.width, w.height, w.nframes, w.rate_px_min, w.null_runs) for t, w in b]
    times = [t for t, _ in a]
    assert times == sorted(times) and times[0] > 0
    for _, w in a:
        assert 8 <= w.nframes <= 120 and 512 <= w.width <= 6000 and 512 <= w.height <= 4000
        assert 0.1 <= w.rate_px_min[0] < w.rate_px_min[1] <= 3.0 and 8 <= w.null_runs <= 32
        span = (w.nframes - 1) * 30.0 / 3600.0
        m = synthetic.motion_count(span, w.rate_px_min[0] * 60, w.rate_px_min[1] * 60, 0.125)
        assert m * w.nframes * w.width * w.height * (1 + w.null_runs) <= 5.0e13
    # without the work bound every draw is kept, in the same order
    c, dc = synthetic.serving_requests(count=5, seed=5, max_adds=None)
    assert dc == 5


def test_bench_reads_profiled_traffic():
    sys.path.insert(0, ROOT)
    import bench
    t4, t1 = bench.profiled_traffic("fullframe-4k"), bench.profiled_traffic("fullframe-1k")
    assert t1 > 0 and t4 == pytest.approx(16 * t1, rel=1e-3)
    assert bench.profiled_traffic("no-such-workload") is None
