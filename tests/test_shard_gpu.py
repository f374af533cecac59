"""Null-run shards on the B200: the shards of a search, run one after another
on one GPU (each an independent call), pool to the unsplit search's null peaks,
threshold, maps and selected peaks."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("count", [2, 3])
def test_shards_pool_to_unsplit_search(device, count):
    import fainttrail_b200 as ftb
    from fainttrail_b200.shard import finish_on_rank0, select_peaks
    g = golden("null_runs_small.npz")
    raw, mjd, exp = g["raw"], g["mjd"], g["exptime"]
    runs = int(g["runs"])
    kw = dict(fwhm_px=2.5, null_runs=runs)
    whole = device.search(raw, mjd, exp, **kw)
    assert whole["threshold"] == float(g["threshold"]) and np.array_equal(whole["null_peaks"], g["pooled"])
    shards = [device.search(raw, mjd, exp, shard_index=k, shard_count=count, **kw) for k in range(count)]
    assert all(s["method"] == "shard" and s["max_snr"] is None for s in shards)
    pooled = np.concatenate([s["null_peaks"] for s in shards])
    assert np.array_equal(pooled, whole["null_peaks"])
    t = ftb.null_threshold(pooled, runs, shards[0]["fwhm"], raw.shape[2], raw.shape[1], shards[0]["n_velocities"],
                           **kw)
    assert t["threshold"] == whole["threshold"] and t["method"] == whole["method"]
    # rank 0's finishing call: the real pass with the pooled threshold given
    fin = finish_on_rank0(device, raw, mjd, exp, t, **kw)
    assert fin["method"] == "calibrated" and fin["threshold"] == whole["threshold"]
    assert np.array_equal(fin["max_snr"], whole["max_snr"]) and fin["peaks"] == whole["peaks"]
    assert fin["selected"] == whole["selected"] == select_peaks(fin["peaks"], t["threshold"], 300)
    assert len(fin["candidates"]) == len(whole["candidates"])
    for (a, fa), (b, fb) in zip(fin["candidates"], whole["candidates"]):
        assert np.array_equal(a, b) and fa == fb


def test_shard_arguments_rejected(device):
    g = golden("null_runs_small.npz")
    with pytest.raises(RuntimeError, match="shard_index"):
        device.search(g["raw"], g["mjd"], g["exptime"], fwhm_px=2.5, shard_index=2, shard_count=2)
    with pytest.raises(RuntimeError, match="fixed threshold"):
        device.search(g["raw"], g["mjd"], g["exptime"], fwhm_px=2.5, threshold_snr=5.0, shard_index=0, shard_count=2)
