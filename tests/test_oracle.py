"""The oracle (CPU restatement under oracle/) pinned against the golden vectors
the reference produced (tests/golden/make_golden.py), and against the
reference build itself where it is present. No GPU."""
import numpy as np
import pytest

from conftest import golden


def same(a, b):
    return np.array_equal(np.asarray(a), np.asarray(b), equal_nan=True)


@pytest.mark.parametrize("name", ["stack_contract.npz", "stack_constant.npz", "stack_nan_table.npz"])
def test_stack_matches_golden(oracle, name):
    g = golden(name)
    dx, dy = oracle.shift_table(g["t_h"], g["vel"])
    ms, bv = oracle.stack(g["frames"], dx, dy, int(g["min_count"]))
    assert same(ms, g["max_snr"]) and same(bv, g["best_v"])
    if "dx" in g:
        ms, bv = oracle.stack(g["frames"], g["dx"], g["dy"], int(g["min_count"]))
        assert same(ms, g["table_max_snr"]) and same(bv, g["table_best_v"])


def test_constant_frames_tie_to_lowest_index(oracle):
    # reference known answer (tests/test_main.cpp:451-456): pixel (18, 11) covered by
    # all 7 frames for every motion; all tie, motion 0 wins with S/N sqrt(7)
    g = golden("stack_constant.npz")
    dx, dy = oracle.shift_table(g["t_h"], g["vel"])
    ms, bv = oracle.stack(g["frames"], dx, dy, 5)
    assert bv[11, 18] == 0
    assert abs(ms[11, 18] - np.sqrt(7.0)) < 1e-5


def test_stage_matches_golden(oracle):
    g = golden("stage_small.npz")
    sub, bgs = oracle.prepare_sub(g["raw"])
    assert same(sub, g["sub"]) and same(bgs, g["background"])
    st = oracle.build_stage(g["sub"], g["t_h"], float(g["fwhm"]))
    for k in ("filtered", "static_sky", "mask", "sigma", "cr"):
        assert same(st[k], g[k]), k


def test_search_pieces_match_golden(oracle):
    g = golden("search_small.npz")
    grid, dv = oracle.velocity_grid(0.18333333340706304, 4.0, 40.0, 0.5)
    assert same(grid, g["grid"]) and dv == float(g["dv"])
    thr, meth, a, k, s2 = oracle.set_threshold(g["null_peaks"].astype(np.float32), 2)
    assert thr == float(g["threshold"]) and meth == 1
    assert (a, k, s2) == (float(g["null_a"]), float(g["null_k"]), float(g["null_inv_s2"]))


def test_median_rules(oracle):
    assert oracle.median([3.0, 1.0, 2.0]) == 2.0
    assert oracle.median([4.0, 1.0, 3.0, 2.0]) == 2.5
    assert oracle.median([]) == 0.0
    assert oracle.robust_sigma([1.0, 2.0]) == 0.0


def test_oracle_against_reference_stage_and_stack(oracle, reference):
    frames, mjd, exp = reference.simulate(width=64, height=48, nframes=10, nstars=30, nmovers=1, seed=3)
    prep = reference.prepare(frames, mjd, exp, fwhm_px=2.5)
    v, im = prep.vectors(), prep.images()
    st = oracle.build_stage(im["sub"], v["t_h"], 2.5)
    assert same(st["filtered"], im["filtered"]) and same(st["static_sky"], im["static_sky"])
    # a permuted (null-run) time order
    t2 = oracle.null_orders(v["t_h"], 1, 99)[0]
    rs = reference.build_stage(im["sub"], t2, 2.5, params=reference.params(fwhm_px=2.5))
    st2 = oracle.build_stage(im["sub"], t2, 2.5)
    for k in ("filtered", "static_sky", "mask", "sigma", "cr"):
        assert same(st2[k], rs[k]), k
    grid, _ = oracle.velocity_grid(prep.span_h, 4.0, 40.0, 0.5)
    dx, dy = oracle.shift_table(v["t_h"], grid)
    mc = oracle.min_count(0.7, prep.n)
    for which in (0, 1, 2):
        ms, bv = reference.stack(st["filtered"], dx=dx, dy=dy, min_count=mc, which=which)
        ms2, bv2 = oracle.stack(st["filtered"], dx, dy, mc)
        assert same(ms, ms2) and same(bv, bv2), which


def test_null_orders_and_peaks_against_reference(oracle, reference):
    t = np.linspace(-0.2, 0.2, 17)
    assert same(oracle.null_orders(t, 4, 12345), reference.null_orders(t, 4, 12345))
    g = golden("search_small.npz")
    rng = np.random.default_rng(1)
    ms = g["max_snr"]
    bv = rng.integers(0, 50, ms.shape).astype(np.int32)
    a = oracle.find_peaks(ms, bv, 3.0, 2, 4, 20000)
    b = reference.find_peaks(ms, bv, 3.0, 2, 4, 20000)
    assert all(same(x, y) for x, y in zip(a, b))
    # plateaus: one peak per plateau, ties ordered as std::sort leaves them
    flat = np.zeros((30, 40), np.float32)
    flat[10:13, 10:14] = 5.0
    flat[20, 30] = 5.0
    a = oracle.find_peaks(flat, np.zeros_like(flat, np.int32), 3.0, 2, 1, 100)
    b = reference.find_peaks(flat, np.zeros_like(flat, np.int32), 3.0, 2, 1, 100)
    assert all(same(x, y) for x, y in zip(a, b)) and len(a[0]) == 2


def _bits_equal(a, b):
    a, b = np.asarray(a, np.float32), np.asarray(b, np.float32)
    na, nb = np.isnan(a), np.isnan(b)
    return np.array_equal(na, nb) and np.array_equal(a.view(np.uint32)[~na], b.view(np.uint32)[~nb])


@pytest.mark.parametrize("n,seed", [(9, 1), (40, 4), (65, 6)])
def test_oracle_stage_signed_zeros_against_reference(oracle, reference, n, seed):
    """Integer-valued frames with +0.0 and -0.0: the restatement's static sky and
    filtered frames equal the reference's bit for bit (equal values ordered by
    time rank, preprocess.cpp:154-204), so the device stage can be held to bits."""
    rng = np.random.default_rng(seed)
    sub = rng.integers(-2, 3, (n, 24, 70)).astype(np.float32)
    sub[(sub == 0) & (rng.random(sub.shape) < 0.5)] = -0.0
    sub[:, :, :2] = np.nan
    t = np.sort(rng.uniform(-0.3, 0.3, n))
    rng.shuffle(t)
    o, r = oracle.build_stage(sub, t, 2.5), reference.build_stage(sub, t, 2.5)
    assert np.signbit(r["static_sky"]).any()
    assert _bits_equal(o["static_sky"], r["static_sky"]) and _bits_equal(o["filtered"], r["filtered"])
