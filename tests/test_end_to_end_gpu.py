"""The reference test suite's end-to-end statistical checks run through the
device search (test_blind_search_recovers and test_null_has_no_detections,
test_main.cpp:216-264): four simulated movers on a 192 x 192 x 40 sequence with
stars, hot pixels and cosmic rays are all recovered blind (PSF width estimated,
registration checked, two null runs) within 4 sigma of their reported errors,
with no false positive; two pure-noise sequences give no detection. The device's
threshold and candidate list are also the reference's on the same frames."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# small_sim and quick_search of the reference's tests (test_main.cpp:63-83)
SMALL = dict(width=192, height=192, nframes=40, exptime_s=45.0, cadence_s=60.0, nstars=200, hot_pixels=15,
             cosmic_rays_per_frame=2.0)
QUICK = dict(vmin_pxh=8.0, vmax_pxh=30.0, null_runs=2)
# x_ref, y_ref, vx_pxh, vy_pxh, mag (test_main.cpp:218-220)
MOVERS = [(40, 50, 22, 10, 18.8), (150, 60, -15, 12, 19.1), (60, 140, 9, -14, 19.3), (140, 150, -12, -18, 19.5)]


def match(cands, truth, max_dpos, max_dv):
    """match (validate.cpp:36-60) over accepted candidates: for each true mover
    in order, the nearest unused candidate within max_dpos and max_dv.
    Returns (truth index, candidate index, position error, motion error)."""
    used = [False] * len(cands)
    out = []
    for t, (x, y, vx, vy, _) in enumerate(truth):
        best, bi, bdv = math.inf, -1, 0.0
        for c, (row, _) in enumerate(cands):
            if used[c] or row[14] == 0:
                continue
            dp = math.hypot(row[0] - x, row[1] - y)
            dv = math.hypot(row[2] - vx, row[3] - vy)
            if dp <= max_dpos and dv <= max_dv and dp < best:
                best, bi, bdv = dp, c, dv
        if bi >= 0:
            used[bi] = True
            out.append((t, bi, best, bdv))
    return out


def _same_as_reference(reference, got, frames, mjd, exp):
    ref = reference.prepare(frames, mjd, exp, **QUICK).search(backend="cpu", **QUICK)
    assert got["threshold"] == ref["threshold"] and got["method"] == ref["method"]
    assert len(got["candidates"]) == len(ref["candidates"])
    for (row, flags), (want, wflags) in zip(got["candidates"], ref["candidates"]):
        assert np.array_equal(row, want) and flags == wflags


def test_blind_search_recovers(device, reference):
    frames, mjd, exp = reference.simulate(movers=MOVERS, seed=3, **SMALL)
    got = device.search(frames, mjd, exp, align="check", **QUICK)
    assert got["registration"]["measured"] == 1 and got["registration"]["registered"] == 1
    assert got["method"] in ("null-fit gauss", "null-fit linear", "null-quantile")
    matched = match(got["candidates"], MOVERS, 1.0, 2.0 * got["dv"] + 1.0)
    assert len(matched) == len(MOVERS)
    for _, ci, dpos, dv in matched:
        row = got["candidates"][ci][0]
        assert dpos < 4.0 * math.sqrt(2.0) * row[4]
        assert dv < 4.0 * math.sqrt(2.0) * row[5] + 0.3
    assert sum(int(row[14]) for row, _ in got["candidates"]) == len(MOVERS)  # no false positive
    _same_as_reference(reference, got, frames, mjd, exp)


@pytest.mark.parametrize("seed", [101, 202])
def test_pure_noise_has_no_detections(device, reference, seed):
    frames, mjd, exp = reference.simulate(seed=seed, nmovers=0, **SMALL)
    got = device.search(frames, mjd, exp, align="check", **QUICK)
    assert sum(int(row[14]) for row, _ in got["candidates"]) == 0
    assert got["threshold"] >= 5.0  # min_snr_floor
    _same_as_reference(reference, got, frames, mjd, exp)
