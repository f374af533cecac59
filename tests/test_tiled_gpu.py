"""The tiled search (ft_b200_search_tiled, search_tiled in tiled.cpp:272-647):
frames kept in host memory and processed in full-width bands with halos must
give exactly the untiled search's result -- detection and argmax maps, real
peaks, pooled null peaks, threshold with its tail fit, every candidate field and
flag -- as the reference's test_tiled_equals_untiled requires of its tiles
(tests/test_main.cpp:1220-1276): band sizes that do and do not divide the
image and one band holding it all, registration-like blank borders that move
with the frame, and registration offsets (the detector test). Both equal the
reference's own search() of the same frames."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def same(a, b):
    assert a["threshold"] == b["threshold"] and a["method"] == b["method"]
    assert (a["null_a"], a["null_k"], a["null_inv_s2"]) == (b["null_a"], b["null_k"], b["null_inv_s2"])
    assert a["fwhm"] == b["fwhm"]
    assert np.array_equal(a["null_peaks"], b["null_peaks"])
    assert np.array_equal(a["max_snr"], b["max_snr"], equal_nan=True)
    assert np.array_equal(a["best_v"], b["best_v"])
    assert a["peaks"] == b["peaks"]
    assert len(a["candidates"]) == len(b["candidates"])
    for (ra, fa), (rb, fb) in zip(a["candidates"], b["candidates"]):
        assert np.array_equal(ra, rb) and fa == fb


def _sequence(reference, seed, w, h, n):
    frames, mjd, exp = reference.simulate(width=w, height=h, nframes=n, nstars=80, nmovers=4, seed=seed,
                                          rate_min_arcsec_min=0.3, rate_max_arcsec_min=1.0)
    for i in range(n):
        frames[i, :, : i % 5] = np.nan  # a blank border that moves with the frame
    reg_dx = -0.5 * (np.arange(n) % 5)
    reg_dy = 0.25 * (np.arange(n) % 3)
    return frames, mjd, exp, reg_dx, reg_dy


@pytest.mark.parametrize("seed,w,h,n,bands", [(31, 160, 130, 16, (48, 100, 1000)), (7, 120, 200, 20, (16, 64))])
def test_tiled_equals_untiled_and_reference(device, reference, seed, w, h, n, bands):
    frames, mjd, exp, reg_dx, reg_dy = _sequence(reference, seed, w, h, n)
    kw = dict(fwhm_px=0.0, null_runs=3, vmin_pxh=5.0, vmax_pxh=40.0, reg_dx=reg_dx, reg_dy=reg_dy)
    untiled = device.search(frames, mjd, exp, **kw)
    for b in bands:
        same(device.search_tiled(frames, mjd, exp, band_rows=b, **kw), untiled)
    rk = {k: v for k, v in kw.items() if not k.startswith("reg_")}
    prep = reference.prepare(frames, mjd, exp, reg_dx=reg_dx, reg_dy=reg_dy, **rk)
    ref = prep.search(backend="cpu", **rk)
    assert untiled["fwhm"] == prep.fwhm and untiled["threshold"] == ref["threshold"]
    assert np.array_equal(untiled["null_peaks"], ref["null_peaks"])
    assert np.array_equal(untiled["max_snr"], ref["max_snr"], equal_nan=True)
    assert len(untiled["candidates"]) == len(ref["candidates"]) > 0
    for (row, flags), (want, wflags) in zip(untiled["candidates"], ref["candidates"]):
        assert np.array_equal(row, want) and flags == wflags


def test_tiled_fixed_threshold_and_bad_arguments(device, reference):
    import fainttrail_b200 as ftb
    frames, mjd, exp, _, _ = _sequence(reference, 5, 96, 90, 12)
    kw = dict(fwhm_px=2.5, threshold_snr=4.0, vmin_pxh=5.0, vmax_pxh=40.0)
    same(device.search_tiled(frames, mjd, exp, band_rows=32, **kw), device.search(frames, mjd, exp, **kw))
    with pytest.raises(RuntimeError, match="band_rows"):
        device.search_tiled(frames, mjd, exp, band_rows=-1, **kw)
    with pytest.raises(RuntimeError, match="frames"):
        device.search_tiled(frames[:3], mjd[:3], exp[:3], band_rows=32, **kw)
