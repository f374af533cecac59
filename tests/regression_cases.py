"""The reference's real-data regression cases as committed fixtures
(tests/golden/regression_<case>.npz, written by tests/golden/make_regression.py):
frames rebuilt from their stored 16-bit integers exactly as the reference's FITS
reader does, with times, registration offsets, search settings and the
reference's search outputs."""
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = ("ceres-cut", "leo-triplet-cut", "mariekebaan-cut")


def load_case(case):
    g = np.load(os.path.join(HERE, "golden", f"regression_{case}.npz"), allow_pickle=False)
    stored = g["stored"].astype(np.float64)
    frames = (g["bzero"][:, None, None] + g["bscale"][:, None, None] * stored).astype(np.float32)
    for i, b in enumerate(g["blank"]):
        if b != np.iinfo(np.int32).min:
            frames[i][g["stored"][i] == b] = np.nan
    flags = json.loads(str(g["flags"]))
    cands = [(g["candidates"][k], flags[k]) for k in range(len(flags))]
    out = {k: g[k] for k in ("mjd", "exptime", "reg_dx", "reg_dy", "null_peaks", "max_snr")}
    out.update(frames=frames, params=json.loads(str(g["params"])), candidates=cands, fwhm=float(g["fwhm"]),
               threshold=float(g["threshold"]), method=str(g["method"]), null_a=float(g["null_a"]),
               null_k=float(g["null_k"]), null_inv_s2=float(g["null_inv_s2"]), n_velocities=int(g["n_velocities"]),
               baseline_threshold=float(g["baseline_threshold"]))
    return out


def same_search(got, want):
    """Bit for bit: PSF width, threshold and tail fit, pooled null peaks,
    detection map, every candidate field and flag."""
    assert got["fwhm"] == want["fwhm"]
    assert got["threshold"] == want["threshold"] and got["method"] == want["method"]
    assert (got["null_a"], got["null_k"], got["null_inv_s2"]) == (want["null_a"], want["null_k"], want["null_inv_s2"])
    assert np.array_equal(got["null_peaks"], want["null_peaks"])
    assert np.array_equal(got["max_snr"], want["max_snr"], equal_nan=True)
    assert len(got["candidates"]) == len(want["candidates"])
    for (row, flags), (wrow, wflags) in zip(got["candidates"], want["candidates"]):
        assert np.array_equal(row, wrow) and flags == wflags
