"""Whole-search parity on the B200 (ft_b200_search): threshold, tail-model
coefficients, pooled null peaks, the real detection map and its peaks against
the reference's own search() (golden vectors, and the reference build live
where it is present)."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def same(a, b):
    return np.array_equal(np.asarray(a), np.asarray(b), equal_nan=True)


def test_golden_search(device, oracle):
    g = golden("search_small.npz")
    r = device.search(g["raw"], g["mjd"], g["exptime"], fwhm_px=2.5, null_runs=2)
    assert r["threshold"] == float(g["threshold"]) and r["method"] == str(g["method"])
    assert (r["null_a"], r["null_k"], r["null_inv_s2"]) == (float(g["null_a"]), float(g["null_k"]),
                                                            float(g["null_inv_s2"]))
    assert same(r["null_peaks"], g["null_peaks"])
    assert same(r["max_snr"], g["max_snr"])
    assert same(r["grid"], g["grid"]) and r["n_velocities"] == int(g["n_velocities"])
    # the real peaks are find_peaks of the map (floor = min_snr_floor 5, radius lround(fwhm))
    px, py, ps, pv = oracle.find_peaks(r["max_snr"], r["best_v"], 5.0, 2, 4, 100000)
    assert [(a, b, c, d) for a, b, c, d in zip(px, py, ps, pv)] == [(x, y, np.float32(s), v) for x, y, s, v in
                                                                 r["peaks"]]
    # refined candidates: all 17 fields of the reference's list, bit for bit
    got = np.array([row for row, _ in r["candidates"]]).reshape(-1, 17)
    assert got.shape == g["candidates"].shape and np.array_equal(got, g["candidates"])


@pytest.mark.parametrize("seed,w,h,n,runs,fwhm", [(21, 160, 128, 24, 3, 2.5), (8, 128, 100, 16, 2, 0.0)])
def test_live_reference_search(device, reference, seed, w, h, n, runs, fwhm):
    R = reference
    frames, mjd, exp = R.simulate(width=w, height=h, nframes=n, nstars=80, nmovers=3, seed=seed,
                                  rate_min_arcsec_min=0.3, rate_max_arcsec_min=0.8)
    frames[:, :, :6] = np.nan  # a blank border, as registered frames have
    prep = R.prepare(frames, mjd, exp, fwhm_px=fwhm, null_runs=runs)
    ref = prep.search(fwhm_px=fwhm, null_runs=runs, backend="cpu")
    got = device.search(frames, mjd, exp, fwhm_px=fwhm, null_runs=runs)
    assert got["fwhm"] == prep.fwhm
    assert got["threshold"] == ref["threshold"] and got["method"] == ref["method"]
    assert same(got["null_peaks"], ref["null_peaks"])
    assert same(got["max_snr"], ref["max_snr"])
    assert len(got["candidates"]) == len(ref["candidates"])
    for (row, flags), (want, wflags) in zip(got["candidates"], ref["candidates"]):
        assert np.array_equal(row, want) and flags == wflags


@pytest.mark.parametrize("seed,nmovers,threshold", [(31, 6, 0.0), (44, 4, 4.0)])
def test_candidates_match_reference(device, reference, seed, nmovers, threshold):
    """Refined candidates on sequences with movers (and, with a low fixed
    threshold, many noise candidates: duplicates, ghosts and flags)."""
    R = reference
    frames, mjd, exp = R.simulate(width=200, height=150, nframes=20, nstars=60, nmovers=nmovers, seed=seed,
                                  rate_min_arcsec_min=0.3, rate_max_arcsec_min=1.5)
    frames[:, :, :5] = np.nan
    kw = dict(fwhm_px=2.5, null_runs=2, threshold_snr=threshold, vmin_pxh=5.0, vmax_pxh=60.0)
    prep = R.prepare(frames, mjd, exp, fwhm_px=2.5, null_runs=2)
    ref = prep.search(backend="cpu", **kw)
    got = device.search(frames, mjd, exp, **kw)
    assert got["threshold"] == ref["threshold"]
    assert len(ref["candidates"]) > 0 and len(got["candidates"]) == len(ref["candidates"])
    for (row, flags), (want, wflags) in zip(got["candidates"], ref["candidates"]):
        assert np.array_equal(row, want) and flags == wflags


def test_fixed_threshold_and_cancel(device):
    import fainttrail_b200 as ftb
    g = golden("search_small.npz")
    r = device.search(g["raw"], g["mjd"], g["exptime"], fwhm_px=2.5, threshold_snr=4.0)
    assert r["method"] == "fixed" and r["threshold"] == 4.0 and len(r["null_peaks"]) == 0
    assert all(s >= 4.0 for _, _, s, _ in r["selected"])
    with pytest.raises(ftb.Cancelled):
        device.search(g["raw"], g["mjd"], g["exptime"], progress=lambda f, s: f < 0.5, fwhm_px=2.5, null_runs=2)
    r2 = device.search(g["raw"], g["mjd"], g["exptime"], fwhm_px=2.5, null_runs=2)
    assert r2["threshold"] == float(g["threshold"])
