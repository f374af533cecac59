"""Null runs split over processes (fainttrail_b200.shard) on the host: the
shard blocks, the all-gather of pooled null peaks over a world-size-2 (and 3)
gloo group, and the threshold every rank computes from the pooled list
(ft_b200_null_threshold, host only), against the reference's own threshold for
the same runs (golden null_runs_small.npz: per-run null peaks of the
reference's search, boundaries from searches with 1..5 runs)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import golden


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_blocks_cover_runs_in_order():
    from fainttrail_b200.shard import shard_block
    for runs in (0, 1, 3, 5, 32, 64):
        for count in (1, 2, 3, 8):
            blocks = [shard_block(runs, k, count) for k in range(count)]
            assert blocks[0][0] == 0 and blocks[-1][1] == runs
            assert all(a[1] == b[0] for a, b in zip(blocks, blocks[1:]))
            assert max(b - a for a, b in blocks) - min(b - a for a, b in blocks) <= 1
    with pytest.raises(ValueError):
        shard_block(4, 2, 2)


def test_null_threshold_matches_reference():
    import fainttrail_b200 as ftb
    g = golden("null_runs_small.npz")
    t = ftb.null_threshold(g["pooled"], int(g["runs"]), float(g["fwhm"]), int(g["width"]), int(g["height"]),
                           int(g["n_velocities"]), fwhm_px=2.5, null_runs=int(g["runs"]))
    assert t["threshold"] == float(g["threshold"]) and t["method"] == str(g["method"])
    assert (t["null_a"], t["null_k"], t["null_inv_s2"]) == (float(g["null_a"]), float(g["null_k"]),
                                                           float(g["null_inv_s2"]))
    s = golden("search_small.npz")
    t2 = ftb.null_threshold(s["null_peaks"], 2, 2.5, 96, 80, int(s["n_velocities"]), fwhm_px=2.5, null_runs=2)
    assert t2["threshold"] == float(s["threshold"])
    # no null runs and no fixed threshold: the Gaussian trial-count rule; a fixed threshold passes through
    assert ftb.null_threshold([], 0, 2.5, 96, 80, 57, threshold_snr=6.5)["method"] == "fixed"


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import fainttrail_b200 as ftb
        from fainttrail_b200.shard import gather_pooled, shard_block
        g = golden("null_runs_small.npz")
        runs = int(g["runs"])
        edges = np.concatenate([[0], np.cumsum(g["run_counts"])])
        k0, k1 = shard_block(runs, rank, world)
        local = g["pooled"][edges[k0]:edges[k1]]  # what this rank's GPU returns for its runs
        pooled = gather_pooled(local)
        t = ftb.null_threshold(pooled, runs, float(g["fwhm"]), int(g["width"]), int(g["height"]),
                               int(g["n_velocities"]), fwhm_px=2.5, null_runs=runs)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), pooled=pooled, threshold=t["threshold"],
                 method=t["method"], k0=k0, k1=k1)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3, 6])  # 6 ranks over 5 runs: one rank has none
def test_gloo_pooled_threshold(tmp_path, world):
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    g = golden("null_runs_small.npz")
    got = [np.load(tmp_path / f"rank{r}.npz") for r in range(world)]
    assert [int(x["k0"]) for x in got] == sorted(int(x["k0"]) for x in got)
    for x in got:
        assert np.array_equal(x["pooled"], g["pooled"])  # rank order = run order
        assert float(x["threshold"]) == float(g["threshold"]) and str(x["method"]) == str(g["method"])
