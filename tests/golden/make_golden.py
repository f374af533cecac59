"""Regenerate the golden fixtures in this directory from the reference itself.

Runs FaintTrail 0.9.1 built from its own sources (oracle/Makefile ->
oracle/_ref/) through oracle/ref_driver.cpp and stores small input/output
vectors as compressed .npz files. Needs the reference build (only where the
reference tree is present); the fixtures it writes are committed, so the tests
that read them run anywhere.

    make -C oracle ref && python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
from ftoracle import Reference  # noqa: E402


def contract_case(R, constant, seed):
    """The awkward pass of the reference's backend contract test
    (tests/test_main.cpp:389-470): 37x23x7, symmetric times with x.5 shifts,
    a 13x13 velocity lattice plus a far-out motion, min_count 5."""
    rng = np.random.default_rng(seed)
    w, h, n = 37, 23, 7
    t = (np.arange(n) - (n - 1) / 2.0) * 0.25
    frames = np.ones((n, h, w), np.float32) if constant else rng.standard_normal((n, h, w)).astype(np.float32)
    vel = [(j * 2.0, k * 2.0) for j in range(-6, 7) for k in range(-6, 7)] + [(400.0, 0.0)]
    vel = np.array(vel)
    ms, bv = R.stack(frames, t_h=t, vel=vel, min_count=5, which=0)
    return dict(frames=frames, t_h=t, vel=vel, min_count=np.int32(5), max_snr=ms, best_v=bv)


def nan_table_case(R, seed):
    """The CUDA-algorithm test pass (tests/test_main.cpp:553-622): 37x23x7 with a
    NaN pixel, 171 motions (far shifts +-400 px) and a curved 150-motion table
    with jumps of +500 / -900 px."""
    rng = np.random.default_rng(seed)
    w, h, n = 37, 23, 7
    t = (np.arange(n) - 3) * 0.25
    frames = rng.standard_normal((n, h, w)).astype(np.float32)
    frames[2].flat[100] = np.nan
    vel = np.array([(j * 2.0, k * 2.0) for j in range(-6, 7) for k in range(-6, 7)] + [(400.0, 0.0), (0.0, -400.0)])
    ms, bv = R.stack(frames, t_h=t, vel=vel, min_count=5, which=0)
    m = 150
    dx = np.zeros((m, n), np.int32)
    dy = np.zeros((m, n), np.int32)
    for j in range(m):
        for i in range(n):
            ti = t[i]
            # np.round is half-to-even; the table uses half away from zero like std::lround
            fx = (j % 13 - 6) * ti + ((j % 7) - 3.0) * ti * ti
            fy = (j % 11 - 5) * ti + ((j % 5) - 2.0) * ti * ti
            dx[j, i] = int(np.sign(fx) * np.floor(abs(fx) + 0.5)) + (500 if j == 77 else 0)
            dy[j, i] = int(np.sign(fy) * np.floor(abs(fy) + 0.5)) - (900 if j == 91 else 0)
    ms2, bv2 = R.stack(frames, dx=dx, dy=dy, min_count=5, which=0)
    return dict(frames=frames, t_h=t, vel=vel, min_count=np.int32(5), max_snr=ms, best_v=bv, dx=dx, dy=dy,
                table_max_snr=ms2, table_best_v=bv2)


def stage_case(R):
    """prepare() on a small simulated sequence: background, blank-border growth,
    static sky, noise, scatter mask, CR rejection, matched filter. Blank (NaN)
    left columns exercise the coverage rule and the grown border."""
    frames, mjd, exp = R.simulate(width=72, height=52, nframes=12, nstars=40, nmovers=2, hot_pixels=6,
                                  cosmic_rays_per_frame=3.0, seed=17)
    frames[:, :, :5] = np.nan
    frames[3, 10:13, 30:33] = np.nan
    prep = R.prepare(frames, mjd, exp, fwhm_px=2.5)
    v, im = prep.vectors(), prep.images()
    return dict(raw=frames, mjd=mjd, exptime=exp, fwhm=np.float64(prep.fwhm), span_h=np.float64(prep.span_h),
                t_h=v["t_h"], sigma=v["sigma"], background=v["background"], cr=v["cr"], sub=im["sub"],
                filtered=im["filtered"], static_sky=im["static_sky"], mask=im["mask"])


def search_case(R):
    """A whole search() with null calibration (2 null runs) on a small sequence:
    threshold, pooled null peaks, detection map and candidates."""
    frames, mjd, exp = R.simulate(width=96, height=80, nframes=12, nstars=60, nmovers=2, seed=5)
    prep = R.prepare(frames, mjd, exp, fwhm_px=2.5, null_runs=2)
    res = prep.search(fwhm_px=2.5, null_runs=2, backend="cpu")
    cands = np.array([c[0] for c in res["candidates"]]).reshape(-1, 17)
    grid, dv = R.velocity_grid(prep.span_h)
    return dict(raw=frames, mjd=mjd, exptime=exp, threshold=np.float64(res["threshold"]),
                method=np.array(res["method"]), null_peaks=res["null_peaks"], max_snr=res["max_snr"],
                n_velocities=np.int32(res["n_velocities"]), dv=np.float64(res["dv"]), candidates=cands,
                null_a=np.float64(res["null_a"]), null_k=np.float64(res["null_k"]),
                null_inv_s2=np.float64(res["null_inv_s2"]), grid=grid)


def null_runs_case(R):
    """The null calibration of a search split by run: 5 null runs on the search
    case's sequence. The permutations come from one seeded stream, so the pooled
    null peaks of k runs are the first part of those of k + 1 runs; the run
    boundaries follow from searches with 1..5 runs. Pins the threshold that
    pooled per-run lists must reproduce, whichever process computed each run."""
    frames, mjd, exp = R.simulate(width=96, height=80, nframes=12, nstars=60, nmovers=2, seed=5)
    runs = 5
    prep = R.prepare(frames, mjd, exp, fwhm_px=2.5, null_runs=runs)
    full = prep.search(fwhm_px=2.5, null_runs=runs, backend="cpu")
    pooled = np.asarray(full["null_peaks"], np.float64)
    counts, prev = [], 0
    for k in range(1, runs + 1):
        part = np.asarray(prep.search(fwhm_px=2.5, null_runs=k, backend="cpu")["null_peaks"], np.float64)
        assert np.array_equal(part, pooled[:part.size]), "pooled null peaks are not run-prefix ordered"
        counts.append(part.size - prev)
        prev = part.size
    assert prev == pooled.size
    return dict(raw=frames, mjd=mjd, exptime=exp, runs=np.int32(runs), pooled=pooled,
                run_counts=np.array(counts, np.int32), threshold=np.float64(full["threshold"]),
                method=np.array(full["method"]), null_a=np.float64(full["null_a"]),
                null_k=np.float64(full["null_k"]), null_inv_s2=np.float64(full["null_inv_s2"]),
                fwhm=np.float64(prep.fwhm), width=np.int32(96), height=np.int32(80),
                n_velocities=np.int32(full["n_velocities"]))


def _shifted(frames, sx, sy):
    """frames[i] moved by (sx[i], sy[i]) whole pixels; uncovered pixels NaN."""
    out = np.full_like(frames, np.nan)
    n, h, w = frames.shape
    for i in range(n):
        dx, dy = int(sx[i]), int(sy[i])
        ys, yd = (slice(0, h - dy), slice(dy, h)) if dy >= 0 else (slice(-dy, h), slice(0, h + dy))
        xs, xd = (slice(0, w - dx), slice(dx, w)) if dx >= 0 else (slice(-dx, w), slice(0, w + dx))
        out[i, yd, xd] = frames[i, ys, xs]
    return out


def registration_case(R):
    """check_registration on simulated sequences (128 x 96, 12 frames, whole ADU):
    registered; drifting by whole pixels; flipped by 180 degrees after the
    meridian from frame 6 on; drifting with blank columns and a blank patch on
    the brightest star; too few stars to tell. Only the first, middle and last
    frame by time take part in the check, so those three (as uint16, NaN where
    the mask says) and their times are stored with the reference's verdict on
    the whole sequence; the verdict on the three alone is asserted equal."""
    out = {}
    names = ["registered", "drift", "flip", "blank", "few"]
    for k, name in enumerate(names):
        frames, mjd, _ = R.simulate(width=128, height=96, nframes=12, nstars=3 if name == "few" else 400,
                                    nmovers=1, hot_pixels=8, cosmic_rays_per_frame=2.0, seed=31 + k)
        frames = np.round(frames).astype(np.float32)
        n = frames.shape[0]
        if name in ("drift", "blank"):
            frames = _shifted(frames, np.round(np.arange(n) * 0.45), np.round(np.arange(n) * -0.3))
        if name == "flip":
            frames[6:] = frames[6:, ::-1, ::-1]
        if name == "blank":
            frames[:, :, :5] = np.nan
            y, x = np.unravel_index(np.nanargmax(frames[0]), frames[0].shape)
            frames[0, max(0, y - 1):y + 2, max(0, x - 1):x + 2] = np.nan
        t = (mjd - mjd[0]) * 24.0
        full = R.check_registration(frames, t)
        pick = [0, n // 2, n - 1]  # times ascend and are distinct
        three = np.ascontiguousarray(frames[pick])
        alone = R.check_registration(three, t[pick])
        assert alone == full, name
        nan = np.isnan(three)
        assert np.all(three[~nan] >= 0) and np.all(three[~nan] <= 65535), "whole ADU must fit uint16"
        out[name + "_frames"] = np.where(nan, 0, three).astype(np.uint16)
        out[name + "_nan"] = np.packbits(nan)
        out[name + "_t"] = t[pick]
        out[name + "_values"] = np.array([full[k] for k in ("measured", "registered", "dx", "dy", "mid_dx",
                                                             "mid_dy", "rate_pxh", "stars", "matched")], np.float64)
        out[name + "_message"] = np.array(full["message"])
    out["names"] = np.array(names)
    return out


CSV_CASES = {
    # name: (simulate arguments, search parameters)
    "null": (dict(width=96, height=80, nframes=12, nstars=60, nmovers=6, seed=21), dict(fwhm_px=2.5, null_runs=2)),
    "fixed": (dict(width=96, height=80, nframes=12, nstars=60, nmovers=4, seed=9),
              dict(fwhm_px=2.5, threshold_snr=3.5)),
}


def candidates_csv_case(R):
    """The reference's candidate file (write_candidates_csv, io.cpp:82-115) of two
    searches: a sequence with six movers and two null runs (candidates with
    false-alarm rates from the null-tail fit), and a sequence with four movers at
    a fixed threshold of S/N 3.5 (more candidates, rejected ones among them). Stored per case: the file's text and the result fields it is
    written from (epoch, threshold, grid, PSF width, the candidates' 17 values and
    flags), the frame times and every candidate's track points in every frame
    (ft_get_track_point), and the simulate() and search arguments (JSON), with
    which the reference's simulate() makes the frames again."""
    import tempfile
    out = {"names": np.array(list(CSV_CASES))}
    for name, (sim, kw) in CSV_CASES.items():
        frames, mjd, exp = R.simulate(**sim)
        prep = R.prepare(frames, mjd, exp, **kw)
        with tempfile.TemporaryDirectory() as tmp:
            res = prep.search(csv_path=os.path.join(tmp, "candidates.csv"), backend="cpu", **kw)
        rows = np.array([c[0] for c in res["candidates"]]).reshape(-1, 17)
        out[name + "_csv"] = np.array(res["candidates_csv"])
        out[name + "_rows"] = rows
        out[name + "_flags"] = np.array([c[1] for c in res["candidates"]] or [""])[:len(res["candidates"])]
        out[name + "_info"] = np.array([res["t_ref_mjd"], res["threshold"], res["dv"], res["fwhm"],
                                        res["n_velocities"]], np.float64)
        out[name + "_method"] = np.array(res["method"])
        out[name + "_setup"] = np.array(json.dumps({"simulate": sim, "search": kw}))
        out[name + "_t_h"] = prep.vectors()["t_h"]
        out[name + "_tracks"] = res["track_points"]
    return out


CASES = {
    "stack_contract": lambda R: contract_case(R, False, 4242),
    "stack_constant": lambda R: contract_case(R, True, 4242),
    "stack_nan_table": lambda R: nan_table_case(R, 99),
    "stage_small": stage_case,
    "search_small": search_case,
    "null_runs_small": null_runs_case,
    "registration_small": registration_case,
    "candidates_csv_small": candidates_csv_case,
}


def main():
    """python make_golden.py [case ...]: the named fixtures, or all of them."""
    R = Reference()
    for name in (sys.argv[1:] or list(CASES)):
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **CASES[name](R))
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
