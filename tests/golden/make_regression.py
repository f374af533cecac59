"""Golden fixtures of the reference's real-data regression cases.

The reference ships three small registered sequences with its regression suite
(tests/regression/{ceres,leo-triplet,mariekebaan}-cut.case, data/*/ *.fits, 16-bit
scaled integers with REGDX / REGDY registration offsets). This script reads each
case's search settings, loads its frames with the reference's own load_frames()
(FaintTrail 0.9.1 built from its sources, oracle/_ref), runs the reference's
prepare() + search() (backend cpu, PSF width estimated, detector test with the
registration offsets), and stores per case, in regression_<case>.npz:

* the stored 16-bit integers of every frame with its BZERO / BSCALE / BLANK, from
  which the frames are rebuilt exactly as the reference's reader does
  (float(BZERO + BSCALE * stored), fits.cpp:337) -- checked here bit for bit
  against load_frames();
* mid-exposure MJD, exposure time, registration offsets;
* the search settings (the case's [search] section over the defaults);
* the reference's outputs: PSF width, threshold and its tail fit, pooled null
  peaks, detection map, and every candidate (17 fields and the flags);
* the threshold of the case's committed baseline file (baselines/<case>.csv).

Needs the reference tree ($FAINTTRAIL_REF, else `reference` beside the
repository) and its build (make -C oracle ref):

    python tests/golden/make_regression.py
"""
import glob
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(HERE))
from ftoracle import Reference  # noqa: E402

CASES = ("ceres-cut", "leo-triplet-cut", "mariekebaan-cut")
SEARCH_KEYS = {"vmin": "vmin_pxh", "vmax": "vmax_pxh", "threshold": "threshold_snr", "null_runs": "null_runs",
               "false_per_run": "target_false_per_run", "fwhm": "fwhm_px", "grid_tol": "grid_tol_px",
               "static_exclude": "static_exclude", "mask_scatter": "mask_scatter",
               "weight_scatter": "weight_scatter", "seed": "seed"}


def reference_root():
    return os.environ.get("FAINTTRAIL_REF") or os.path.join(os.path.dirname(ROOT), "reference")


def case_settings(path):
    """The [search] section of a .case file as search keyword arguments."""
    out, section = {}, ""
    for line in open(path):
        line = line.split("#", 1)[0].strip()
        if not line:
            continue
        if line.startswith("["):
            section = line.strip("[]").split()[0]
            continue
        if section == "search" and "=" in line:
            k, v = (x.strip() for x in line.split("=", 1))
            if k in SEARCH_KEYS:
                out[SEARCH_KEYS[k]] = int(v) if k in ("null_runs", "static_exclude", "seed") else float(v)
    return out


def read_fits16(path):
    """A 16-bit FITS image: (stored int16 array, bzero, bscale, blank or None)."""
    raw = open(path, "rb").read()
    cards, off = {}, 0
    while True:
        block = raw[off:off + 2880].decode("ascii")
        off += 2880
        done = False
        for k in range(0, 2880, 80):
            card = block[k:k + 80]
            key = card[:8].strip()
            if key == "END":
                done = True
                break
            if card[8:10] == "= ":
                cards[key] = card[10:].split("/", 1)[0].strip().strip("'").strip()
        if done:
            break
    assert int(cards["BITPIX"]) == 16 and int(cards["NAXIS"]) == 2
    w, h = int(cards["NAXIS1"]), int(cards["NAXIS2"])
    data = np.frombuffer(raw[off:off + 2 * w * h], dtype=">i2").reshape(h, w).astype(np.int16)
    blank = int(cards["BLANK"]) if "BLANK" in cards else None
    return data, float(cards.get("BZERO", 0.0)), float(cards.get("BSCALE", 1.0)), blank


def rebuild(stored, bzero, bscale, blank):
    """float(BZERO + BSCALE * stored) per frame, NaN where BLANK (fits.cpp:331-337)."""
    v = stored.astype(np.float64)
    out = (bzero[:, None, None] + bscale[:, None, None] * v).astype(np.float32)
    if blank is not None:
        for i, b in enumerate(blank):
            if b != np.iinfo(np.int32).min:
                out[i][stored[i] == b] = np.nan
    return out


def baseline_threshold(path):
    for line in open(path):
        m = re.search(r"threshold_snr=([0-9.]+)", line)
        if m:
            return float(m.group(1))
    return float("nan")


def main():
    R = Reference()
    reg_dir = os.path.join(reference_root(), "tests", "regression")
    for case in CASES:
        files = sorted(glob.glob(os.path.join(reg_dir, "data", case, "*.fits")))
        loaded = R.load_frames(files)
        parts = [read_fits16(f) for f in files]
        stored = np.stack([p[0] for p in parts])
        bzero = np.array([p[1] for p in parts])
        bscale = np.array([p[2] for p in parts])
        blank = np.array([p[3] if p[3] is not None else np.iinfo(np.int32).min for p in parts], np.int64)
        frames = rebuild(stored, bzero, bscale, blank)
        a, b = frames, loaded["frames"]
        assert np.array_equal(np.isnan(a), np.isnan(b))
        assert np.array_equal(a.view(np.uint32)[~np.isnan(a)], b.view(np.uint32)[~np.isnan(b)]), case
        assert loaded["reg_dx"] is not None
        kw = case_settings(os.path.join(reg_dir, case + ".case"))
        prep = R.prepare(frames, loaded["mjd"], loaded["exptime"], reg_dx=loaded["reg_dx"], reg_dy=loaded["reg_dy"],
                         **kw)
        res = prep.search(backend="cpu", **kw)
        cands = np.array([row for row, _ in res["candidates"]]).reshape(-1, 17)
        flags = json.dumps([f for _, f in res["candidates"]])
        base = baseline_threshold(os.path.join(reg_dir, "baselines", case + ".csv"))
        out = os.path.join(HERE, f"regression_{case}.npz")
        np.savez_compressed(out, stored=stored, bzero=bzero, bscale=bscale, blank=blank, mjd=loaded["mjd"],
                            exptime=loaded["exptime"], reg_dx=loaded["reg_dx"], reg_dy=loaded["reg_dy"],
                            params=json.dumps(kw), fwhm=prep.fwhm, threshold=res["threshold"],
                            method=res["method"], null_a=res["null_a"], null_k=res["null_k"],
                            null_inv_s2=res["null_inv_s2"], null_peaks=res["null_peaks"], max_snr=res["max_snr"],
                            n_velocities=res["n_velocities"], candidates=cands, flags=flags,
                            baseline_threshold=base)
        print(f"{case}: {frames.shape}, fwhm {prep.fwhm:.3f}, threshold {res['threshold']:.4f} "
              f"({res['method']}; baseline {base}), {len(res['null_peaks'])} null peaks, "
              f"{len(res['candidates'])} candidates -> {os.path.basename(out)} ({os.path.getsize(out) >> 10} KB)")


if __name__ == "__main__":
    main()
