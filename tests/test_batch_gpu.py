"""Batched search with injection-recovery copies (ft_b200_search_batch) against
the reference: each copy must equal the reference's inject() + prepare() +
search() with the calibrated threshold held fixed and no null runs (the searches
completeness() runs, validate.cpp:88-126); the batch's own search must equal a
plain ft_b200_search."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def same(a, b):
    return np.array_equal(np.asarray(a), np.asarray(b), equal_nan=True)


def test_copies_match_reference_inject_and_search(device, reference, oracle):
    R = reference
    frames, mjd, exp = R.simulate(width=128, height=100, nframes=16, nstars=60, nmovers=1, seed=33,
                                  rate_min_arcsec_min=0.3, rate_max_arcsec_min=0.8)
    kw = dict(fwhm_px=2.5, null_runs=2, vmin_pxh=8.0, vmax_pxh=30.0)
    copies = [[(40.0, 50.0, 20.0, -9.0, 900.0), (90.0, 30.0, -14.0, 12.0, 500.0)],
              [(64.5, 70.25, 11.0, 15.0, 1200.0)],
              []]
    base, outs = device.search_batch(frames, mjd, exp, copies, **kw)
    plain = device.search(frames, mjd, exp, **kw)
    assert base["threshold"] == plain["threshold"] and same(base["null_peaks"], plain["null_peaks"])
    assert same(base["max_snr"], plain["max_snr"]) and base["peaks"] == plain["peaks"]
    prep = R.prepare(frames, mjd, exp, fwhm_px=2.5, null_runs=2)
    ref = prep.search(backend="cpu", **kw)
    assert base["threshold"] == ref["threshold"]
    t_ref = 0.5 * (mjd[0] + mjd[-1])
    for objs, got in zip(copies, outs):
        injected = R.inject(frames, mjd, exp, np.array(objs, np.float64).reshape(-1, 5), t_ref, 2.5)
        p2 = R.prepare(injected, mjd, exp, fwhm_px=2.5)
        want = p2.search(backend="cpu", fwhm_px=2.5, vmin_pxh=8.0, vmax_pxh=30.0, null_runs=0,
                         threshold_snr=ref["threshold"])
        assert got["method"] == "fixed" and got["threshold"] == ref["threshold"]
        assert same(got["max_snr"], want["max_snr"])
        assert len(got["candidates"]) == len(want["candidates"])
        for (row, flags), (wrow, wflags) in zip(got["candidates"], want["candidates"]):
            assert np.array_equal(row, wrow) and flags == wflags
        px, py, ps, pv = oracle.find_peaks(got["max_snr"], got["best_v"], np.float32(ref["threshold"]), 2, 4, 100000)
        assert got["peaks"] == [(int(a), int(b), float(c), int(d)) for a, b, c, d in zip(px, py, ps, pv)]


def test_launch_cap_and_device_frames(device):
    """One pass per launch (passes_per_launch 1, the plain path) and the batch
    over device-resident frames give the same results as the batched host call."""
    import torch
    from conftest import golden
    g = golden("search_small.npz")
    raw, mjd, exp = g["raw"], g["mjd"], g["exptime"]
    n, h, w = raw.shape
    copies = [[(30.0, 40.0, 20.0, -9.0, 900.0)], [(50.5, 20.25, -11.0, 15.0, 1200.0), (20.0, 20.0, 5.0, 5.0, 700.0)]]
    kw = dict(fwhm_px=2.5, null_runs=3)
    base, outs = device.search_batch(raw, mjd, exp, copies, **kw)
    base1, outs1 = device.search_batch(raw, mjd, exp, copies, passes_per_launch=1, **kw)
    base2, outs2 = device.search_batch(raw, mjd, exp, copies, passes_per_launch=2, **kw)
    d = torch.from_numpy(np.ascontiguousarray(raw)).cuda()
    base3, outs3 = device.search_batch_dev(d.data_ptr(), w, h, w, n, mjd, exp, copies, **kw)
    for b, o in ((base1, outs1), (base2, outs2), (base3, outs3)):
        assert b["threshold"] == base["threshold"] and same(b["null_peaks"], base["null_peaks"])
        assert same(b["max_snr"], base["max_snr"]) and same(b["best_v"], base["best_v"])
        assert b["peaks"] == base["peaks"]
        for x, y in zip(o, outs):
            assert same(x["max_snr"], y["max_snr"]) and x["peaks"] == y["peaks"]
    one = device.search(raw, mjd, exp, passes_per_launch=1, **kw)
    assert one["threshold"] == base["threshold"] and same(one["max_snr"], base["max_snr"])


def test_completeness_matches_reference(device, reference):
    """completeness() end to end: the calibrated threshold, the seeded placements,
    every level's copy search and the matching -- each row, the baseline count and
    the interpolated S/N at 50 % equal the reference's."""
    import fainttrail_b200 as ftb
    R = reference
    frames, mjd, exp = R.simulate(width=200, height=150, nframes=16, nstars=60, nmovers=2, seed=12,
                                  rate_min_arcsec_min=0.3, rate_max_arcsec_min=1.2)
    kw = dict(fwhm_px=2.5, null_runs=2, vmin_pxh=5.0, vmax_pxh=50.0)
    args = ([4.0, 7.0, 9.0, 12.0], 5, 30.0, 7)
    want = R.completeness(frames, mjd, exp, *args, **kw)
    got = ftb.completeness(device, frames, mjd, exp, snr_levels=args[0], per_level=args[1], min_separation=args[2],
                           seed=args[3], **kw)
    assert got["threshold"] == want["threshold"] and got["method"] == want["method"]
    assert got["baseline_ok"] == want["baseline_ok"] and got["snr50"] == want["snr50"]
    assert sum(r["injected"] for r in want["rows"]) > 0 and sum(r["recovered"] for r in want["rows"]) > 0
    for g, r in zip(got["rows"], want["rows"]):
        assert g == {k: (type(g[k])(v)) for k, v in r.items()}
