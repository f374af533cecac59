"""Parity of the device search with the reference's own search() at the sizes of
the benchmark configurations, on the same seeded synthetic frames.

* The plain CPU-runnable search in full: 20 x 1024^2 frames, 60 s cadence, rates
  0.2-1.1 px/min on a half-pixel grid (5,468 trial motions), 8 null runs.
* The full-frame 4096^2 sequence (40 frames, 30 s cadence, 19,328 motions)
  cropped to the 512 x 512 window the CPU baseline times, with its 3 null runs.
* The large-sensor sequence (60 x 9576 x 6388) cut to a 256 x 256 crop with 2
  null runs, through the tiled path in 64-row bands.
* The batched calibration sequence (30 frames, 2048^2) cut to a 512 x 512 crop
  with 8 null runs and 2 injection copies of 50 objects each, against the
  reference's inject() + prepare() + search() per copy (validate.cpp:88-126).

Everything is compared bit for bit: the threshold and its tail fit (a, k,
inv_s2), the pooled null peaks, the detection map max_snr, the argmax map best_v
(against the reference CPU backend's pass over the reference's own prepared
frames: backend_cpu.cpp:77-204), the real pass's peaks (find_peaks,
search.cpp:105-135) and every field and flag of the refined candidates. The
reference runs on every host core (OpenMP), the device search on cuda:0.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def same(a, b):
    return np.array_equal(np.asarray(a), np.asarray(b), equal_nan=True)


def _frames(name, seed, crop=None):
    import torch
    from fainttrail_b200 import synthetic
    wl = synthetic.WORKLOADS[name]
    frames, mjd, exptime, _ = synthetic.generate(wl, seed=seed, device="cuda")
    if crop:
        frames = frames[:, :crop, :crop]
    host = np.ascontiguousarray(frames.cpu().numpy())
    del frames
    torch.cuda.empty_cache()
    return wl, host, mjd, exptime


def _compare_search(R, device, frames, mjd, exptime, params, min_peaks=1, search=None):
    prep = R.prepare(frames, mjd, exptime, fwhm_px=params["fwhm_px"], null_runs=params["null_runs"])
    ref = prep.search(backend="cpu", **params)
    got = (search or device.search)(frames, mjd, exptime, **params)
    assert got["fwhm"] == prep.fwhm and got["n_velocities"] == ref["n_velocities"]
    assert got["threshold"] == ref["threshold"] and got["method"] == ref["method"]
    assert (got["null_a"], got["null_k"], got["null_inv_s2"]) == (ref["null_a"], ref["null_k"], ref["null_inv_s2"])
    assert len(ref["null_peaks"]) >= min_peaks and same(got["null_peaks"], ref["null_peaks"])
    assert same(got["max_snr"], ref["max_snr"])
    # best_v: the reference CPU backend's real pass over the reference's prepared frames
    v = prep.vectors()
    grid = got["grid"]
    mc = max(3, int(np.ceil(0.7 * prep.n)))
    ms_cpu, bv_cpu = R.stack(prep.images()["filtered"], t_h=v["t_h"], vel=grid, min_count=mc)
    assert same(ms_cpu, ref["max_snr"]) and same(got["best_v"], bv_cpu)
    # the real pass's peaks: find_peaks with the search's floor (min_snr_floor 5
    # under a calibrated threshold), radius max(2, lround(fwhm)), edge 4, at most
    # 100,000 (search.cpp:746-753)
    radius = max(2, int(np.floor(prep.fwhm + 0.5)))
    floor = np.float32(params.get("threshold_snr", 0.0) or 5.0)
    px, py, ps, pv = R.find_peaks(ref["max_snr"], bv_cpu, floor, radius, 4, 100000)
    want_peaks = [(int(a), int(b), float(c), int(d)) for a, b, c, d in zip(px, py, ps, pv)]
    got_peaks = [(int(a), int(b), float(c), int(d)) for a, b, c, d in got["peaks"]]
    assert got_peaks == want_peaks
    assert len(got["candidates"]) == len(ref["candidates"])
    for (row, flags), (want, wflags) in zip(got["candidates"], ref["candidates"]):
        assert np.array_equal(row, want) and flags == wflags
    return got, ref


def test_plain_1k_search_in_full(device, reference):
    """The plain CPU-runnable configuration at its full size, seed 7."""
    wl, frames, mjd, exptime = _frames("plain-1k", 7)
    params = wl.search_params()
    got, ref = _compare_search(reference, device, frames, mjd, exptime, params, min_peaks=100)
    assert got["n_velocities"] == 5468 and len(got["candidates"]) > 0


def test_fullframe_4k_crop(device, reference):
    """The full-frame 4096^2 sequence, 512 x 512 crop, the whole 19,328-motion grid."""
    wl, frames, mjd, exptime = _frames("fullframe-4k", 7, crop=512)
    got, _ = _compare_search(reference, device, frames, mjd, exptime, wl.search_params(), min_peaks=100)
    assert got["n_velocities"] == 19328


def test_large_sensor_crop_tiled(device, reference):
    """The large-sensor sequence (60 x 9576 x 6388 frames, 30 s cadence, rates
    0.05-3 px/min: 98,948 trial motions), a 256 x 256 crop with 2 null runs,
    searched by the tiled path (ft_b200_search_tiled) in 64-row bands."""
    wl, frames, mjd, exptime = _frames("large-sensor", 7, crop=256)
    params = dict(wl.search_params(), null_runs=2)
    got, _ = _compare_search(reference, device, frames, mjd, exptime, params, min_peaks=10,
                             search=lambda f, m, e, **kw: device.search_tiled(f, m, e, band_rows=64, **kw))
    assert got["n_velocities"] == 98948


def test_batched_2k_crop_with_injection_copies(device, reference, oracle):
    """The batched calibration sequence on a 512 x 512 crop: 8 null runs and two
    injection copies of 50 objects, batched on the device, each copy against the
    reference's inject() + prepare() + search() at the calibrated threshold."""
    from fainttrail_b200 import synthetic
    R = reference
    wl, frames, mjd, exptime = _frames("batched-2k", 7, crop=512)
    params = dict(wl.search_params(), null_runs=8)
    copies = synthetic.injection_copies(wl, frames.shape, seed=11)[:2]
    assert len(copies) == 2 and all(len(c) == 50 for c in copies)
    base, outs = device.search_batch(frames, mjd, exptime, copies, **params)
    prep = R.prepare(frames, mjd, exptime, fwhm_px=params["fwhm_px"], null_runs=8)
    ref = prep.search(backend="cpu", **params)
    assert base["threshold"] == ref["threshold"] and base["method"] == ref["method"]
    assert same(base["null_peaks"], ref["null_peaks"]) and same(base["max_snr"], ref["max_snr"])
    assert len(base["candidates"]) == len(ref["candidates"])
    for (row, flags), (want, wflags) in zip(base["candidates"], ref["candidates"]):
        assert np.array_equal(row, want) and flags == wflags
    t_ref = 0.5 * (mjd[0] + mjd[-1])
    recovered = 0
    for objs, got in zip(copies, outs):
        injected = R.inject(frames, mjd, exptime, np.array(objs, np.float64).reshape(-1, 5), t_ref, params["fwhm_px"])
        p2 = R.prepare(injected, mjd, exptime, fwhm_px=params["fwhm_px"])
        want = p2.search(backend="cpu", **dict(params, null_runs=0, threshold_snr=ref["threshold"]))
        assert got["method"] == "fixed" and got["threshold"] == ref["threshold"]
        assert same(got["max_snr"], want["max_snr"])
        assert len(got["candidates"]) == len(want["candidates"])
        for (row, flags), (wrow, wflags) in zip(got["candidates"], want["candidates"]):
            assert np.array_equal(row, wrow) and flags == wflags
        recovered += len(want["candidates"])
    assert recovered > 0
