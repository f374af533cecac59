"""A search's null runs split over GPUs, one process per GPU.

The null runs of a search (FaintTrail search.cpp:757-785) are independent: each
permutes the frame times, rebuilds the preprocessing, stacks and screens its
peaks. Rank k of N runs the block [runs*k/N, runs*(k+1)/N) with the permutations
an unsplit search gives those runs (one seeded stream, search.cpp:559-571), and
the one exchange is the pooled null-peak S/N lists (at most 20,000 values per
run, pool_null_peaks, search.cpp:690-693): every rank all-gathers them in rank
order, which is run order, and computes the same threshold from the
concatenation (set_threshold, search.cpp:573-612), so no broadcast is needed.
Rank 0 then runs the real pass with that threshold given (calibrated_threshold):
its peaks, the selection (select_peaks, search.cpp:614-620) and the refined
candidates. The result equals the unsplit search bit for bit.

The exchange runs over whatever process group the caller passes: NCCL between
GPUs (tensors on the current device) or gloo on the host.
"""
import numpy as np


def shard_block(runs, index, count):
    """The null runs shard `index` of `count` computes: [k0, k1)."""
    if count < 1 or not 0 <= index < count:
        raise ValueError("shard index out of range")
    return runs * index // count, runs * (index + 1) // count


def gather_pooled(local, group=None):
    """All-gather every rank's pooled null-peak S/N values (float64 arrays of
    any length) and concatenate them in rank order."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else \
        torch.device("cpu")
    local = np.ascontiguousarray(local, dtype=np.float64)
    n = torch.tensor([local.size], dtype=torch.int64, device=dev)
    sizes = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(sizes, n, group=group)
    sizes = [int(s.item()) for s in sizes]
    cap = max(1, max(sizes))
    buf = torch.zeros(cap, dtype=torch.float64, device=dev)
    buf[:local.size] = torch.from_numpy(local).to(dev)
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    return np.concatenate([p[:s].cpu().numpy() for p, s in zip(parts, sizes)])


def select_peaks(peaks, threshold, max_candidates):
    """select_peaks (search.cpp:614-620): peaks at or above the threshold with a
    motion, in their order, at most max_candidates."""
    keep = [pk for pk in peaks if float(pk[2]) >= threshold and pk[3] >= 0]
    return keep[:max_candidates]


def sharded_search(dev, frames, mjd, exptime, group=None, **kw):
    """One search with its null runs split over the ranks of `group`; every rank
    calls it with the same frames and parameters. Returns the search result on
    rank 0 (maps, peaks, threshold and tail fit, pooled null peaks, selected
    peaks, candidates) and, on the other ranks, their shard's result with the
    common threshold."""
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    runs = kw.get("null_runs", 3)
    r = dev.search(frames, mjd, exptime, shard_index=rank, shard_count=world, **kw)
    pooled = gather_pooled(r["null_peaks"], group)
    n, h, w = np.shape(frames)
    thr = null_threshold_for(r, pooled, runs, w, h, **kw)
    if rank == 0:
        r = finish_on_rank0(dev, frames, mjd, exptime, thr, **kw)
    r.update(thr)
    r["null_peaks"] = pooled
    return r


def finish_on_rank0(dev, frames, mjd, exptime, thr, **kw):
    """The real pass, its peaks, selection and candidates with the pooled
    threshold and tail fit given."""
    return dev.search(frames, mjd, exptime, calibrated_threshold=thr["threshold"],
                      calibrated_tail=(thr["null_a"], thr["null_b"], thr["null_k"], thr["null_inv_s2"]), **kw)


def null_threshold_for(result, pooled, runs, width, height, **kw):
    """The threshold of a search whose pooled null peaks are `pooled`, with the
    PSF width and motion count of one of its shard results."""
    from . import null_threshold
    return null_threshold(pooled, runs, result["fwhm"], width, height, result["n_velocities"], **kw)
