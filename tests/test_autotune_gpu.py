"""The tile-shape autotuner on a pass large enough to be tuned (30 frames of
2048 x 1024, 12,604 motions: 7.9e11 adds): it caches a shape for the pass's
(frames, motions, width, height), and the maps do not depend on the shape
(automatic, 32 x 16 and 64 x 8 paired tiles give the same bits)."""
import dataclasses

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_autotuned_pass_equals_fixed_shapes(device):
    import fainttrail_b200 as ftb
    from fainttrail_b200 import synthetic
    wl = dataclasses.replace(synthetic.WORKLOADS["batched-2k"], name="tune", height=1024, nmovers=4, null_runs=0)
    frames, mjd, exptime, _ = synthetic.generate(wl, seed=3, device="cuda")
    n, h, w = frames.shape
    kw = dict(wl.search_params(), threshold_snr=6.0)
    ftb.clear_tuned_shapes()
    out = {}
    try:
        for shape in (0, 1, 2):
            ftb.set_tile_shape(shape)
            out[shape] = device.search_dev(frames.data_ptr(), w, h, w, n, mjd, exptime, **kw)
    finally:
        ftb.set_tile_shape(0)
    tuned = ftb.tuned_shapes()
    m = out[0]["n_velocities"]
    assert tuned.get((n, m, w, h)) in range(1, 9)  # a compiled shape that fits
    for shape in (1, 2):
        assert np.array_equal(out[shape]["max_snr"], out[0]["max_snr"])
        assert np.array_equal(out[shape]["best_v"], out[0]["best_v"])
        assert out[shape]["peaks"] == out[0]["peaks"]
