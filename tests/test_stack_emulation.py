"""The stacking kernel's plan checked without a GPU, as the reference checks its
CUDA algorithm by host emulation (test_cuda_algorithm, test_main.cpp:553-622):
ft_b200_emulate_stack plans a pass exactly as the device does for each kernel
shape and walks the plan on the CPU (windows zero-filled outside the frame,
16-bit offsets, coverage counts with the interior-tile shortcut, the maximum
rule); its maps must equal the oracle's and the reference's golden maps bit for
bit: the backend-contract passes (ties, far motions), NaN pixels, shift tables
with +500 / -900 px jumps, random lattices up to 255 frames, every min_count
including ones above the frame count."""
import numpy as np
import pytest

import fainttrail_b200 as ftb
from conftest import golden

SHAPES = range(1, 9)


def same(a, b):
    return np.array_equal(a, b, equal_nan=True)


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("name", ["stack_contract", "stack_constant", "stack_nan_table"])
def test_golden_passes(oracle, name, shape):
    g = golden(name + ".npz")
    dx, dy = oracle.shift_table(g["t_h"], g["vel"])
    ms, bv = ftb.emulate_stack(g["frames"], dx, dy, int(g["min_count"]), shape)
    assert same(ms, g["max_snr"]) and np.array_equal(bv, g["best_v"])
    if "dx" in g:  # the curved table with jumps
        ms, bv = ftb.emulate_stack(g["frames"], g["dx"], g["dy"], int(g["min_count"]), shape)
        assert same(ms, g["table_max_snr"]) and np.array_equal(bv, g["table_best_v"])


def test_constant_frames_tie_to_motion_zero(oracle):
    """The known answer of the reference's contract test (test_main.cpp:451-456):
    constant frames tie every motion; pixel (18, 11) goes to motion 0 with S/N
    sqrt(7), in every tile shape."""
    g = golden("stack_constant.npz")
    dx, dy = oracle.shift_table(g["t_h"], g["vel"])
    for shape in SHAPES:
        ms, bv = ftb.emulate_stack(g["frames"], dx, dy, int(g["min_count"]), shape)
        assert bv[11, 18] == 0 and ms[11, 18] == np.float32(np.sqrt(7.0)), shape


@pytest.mark.parametrize("n,w,h,m,seed,shape", [
    (5, 37, 23, 30, 1, 1), (9, 41, 29, 60, 2, 2), (12, 70, 33, 45, 3, 3), (16, 65, 20, 40, 4, 4),
    (7, 100, 50, 80, 5, 5), (11, 33, 47, 25, 6, 6), (6, 64, 36, 50, 7, 7), (40, 48, 24, 20, 8, 0),
    (120, 40, 20, 12, 9, 0), (255, 36, 12, 6, 10, 0)])
def test_random_lattices(oracle, n, w, h, m, seed, shape):
    rng = np.random.default_rng(seed)
    frames = rng.normal(0, 1, (n, h, w)).astype(np.float32)
    frames[rng.integers(0, n), rng.integers(0, h), rng.integers(0, w)] = np.nan
    frames[:, 3, :] = np.round(frames[:, 3, :])  # integer values: exact ties
    span = rng.integers(1, 60)
    dx = rng.integers(-span, span + 1, (m, n)).astype(np.int32)
    dy = rng.integers(-span, span + 1, (m, n)).astype(np.int32)
    dx[0, :] = 0
    dy[0, :] = 0
    for min_count in sorted({1, max(1, n // 2), n, n + 1}):
        want = oracle.stack(frames, dx, dy, min_count)
        got = ftb.emulate_stack(frames, dx, dy, min_count, shape)
        assert same(got[0], want[0]) and np.array_equal(got[1], want[1]), min_count


def test_min_count_above_frame_count_defines_nothing(oracle):
    rng = np.random.default_rng(11)
    frames = rng.normal(0, 1, (5, 23, 37)).astype(np.float32)
    d = np.zeros((3, 5), np.int32)
    ms, bv = ftb.emulate_stack(frames, d, d, 6, 1)
    assert not ms.any() and np.all(bv == -1)
    want = oracle.stack(frames, d, d, 6)
    assert same(ms, want[0]) and np.array_equal(bv, want[1])


def test_bad_arguments_are_errors():
    f = np.zeros((3, 8, 8), np.float32)
    d = np.zeros((1, 3), np.int32)
    with pytest.raises(RuntimeError, match="min_count"):
        ftb.emulate_stack(f, d, d, 0)
    with pytest.raises(RuntimeError, match="tile shape"):
        ftb.emulate_stack(f, d, d, 1, shape=9)


def test_headline_motion_grid(oracle):
    """The motion grid of the 40-frame full-frame benchmark (0.325 h span, 6-120
    px/h, 0.125 px tolerance: 19,328 motions) on a 64 x 64 crop: the large
    groups the planner builds for it reproduce the oracle's maps."""
    n = 40
    t = np.linspace(-0.1625, 0.1625, n)
    grid, _ = oracle.velocity_grid(0.325, 6.0, 120.0, 0.125)
    assert grid.shape[0] == 19328
    dx, dy = oracle.shift_table(t, grid)
    frames = np.random.default_rng(12).normal(0, 1, (n, 64, 64)).astype(np.float32)
    mc = oracle.min_count(0.7, n)
    got = ftb.emulate_stack(frames, dx, dy, mc)
    want = oracle.stack(frames, dx, dy, mc)
    assert same(got[0], want[0]) and np.array_equal(got[1], want[1])


def test_seeded_random_passes(oracle):
    """400 seeded random passes: 1-255 frames, 1-119 x 1-79 pixels, up to 300
    motions with shifts of 3 to 1000 px (random or straight-track tables),
    integer-valued ties, NaN, +-inf and near-overflow pixels, every min_count up
    to n + 1 and every tile shape."""
    rng = np.random.default_rng(2026)
    for case in range(400):
        n = int(rng.choice([1, 2, 3, 5, 8, 13, 30, 64, 100, 255]))
        w, h = int(rng.integers(1, 120)), int(rng.integers(1, 80))
        m = int(rng.integers(1, 300 if n * w * h < 20000 else 40))
        span = int(rng.choice([3, 40, 400, 1000]))
        if rng.random() < 0.3:  # straight tracks: round(v t) half away from zero
            t = np.sort(rng.uniform(-0.5, 0.5, n))
            f = rng.uniform(-span, span, (m, 2))[:, None, :] * t[None, :, None]
            r = (np.sign(f) * np.floor(np.abs(f) + 0.5)).astype(np.int32)
            dx, dy = np.ascontiguousarray(r[:, :, 0]), np.ascontiguousarray(r[:, :, 1])
        else:
            dx = rng.integers(-span, span + 1, (m, n)).astype(np.int32)
            dy = rng.integers(-span, span + 1, (m, n)).astype(np.int32)
        frames = rng.normal(0, 1, (n, h, w)).astype(np.float32)
        if rng.random() < 0.5:
            frames = np.round(frames)
        if rng.random() < 0.4:
            k = int(rng.integers(1, 6))
            frames.flat[rng.integers(0, frames.size, k)] = rng.choice(
                [np.inf, -np.inf, np.nan, 3e38, -3e38], k).astype(np.float32)
        mc, shape = int(rng.integers(1, n + 2)), int(rng.integers(0, 8))
        got = ftb.emulate_stack(frames, dx, dy, mc, shape)
        want = oracle.stack(frames, dx, dy, mc)
        assert same(got[0], want[0]) and np.array_equal(got[1], want[1]), (case, n, w, h, m, span, mc, shape)


@pytest.mark.parametrize("grid_tol,n,w,h,shape", [(0.125, 20, 96, 70, 1), (0.125, 40, 70, 50, 7), (0.5, 12, 80, 64, 3),
                                                  (0.5, 30, 64, 40, 4), (0.3, 25, 90, 45, 0)])
def test_lattice_blocks_share_columns(oracle, grid_tol, n, w, h, shape):
    """Velocity lattices (the search's own grids, velocity_grid's rule) are
    planned in blocks of motions that share their column in every frame, read
    through row descriptors with row offsets up to 3 (grid_tol 0.5 spreads four
    motions over three rows at the ends of the sequence); the plan, walked on
    the CPU, equals the oracle bit for bit, border tiles included."""
    rng = np.random.default_rng(n)
    t = np.sort(rng.uniform(0.0, 1.5, n))
    t = t - 0.5 * (t[0] + t[-1])
    grid, _ = oracle.velocity_grid(t[-1] - t[0], 2.0, 24.0, grid_tol)
    dx, dy = oracle.shift_table(t, grid)
    st = ftb.plan_stats(w, h, n, dx, dy, shape)
    assert st["row_groups"] == st["groups"] and st["pads"] * 10 < st["slots"]
    frames = rng.normal(0, 1, (n, h, w)).astype(np.float32)
    frames[:, 5, :] = np.round(frames[:, 5, :])  # exact ties
    frames[1, 7, 9] = np.nan
    for mc in (max(1, int(np.ceil(0.7 * n))), n):
        ms, bv = ftb.emulate_stack(frames, dx, dy, mc, shape)
        want_ms, want_bv = oracle.stack(frames, dx, dy, mc)
        assert same(ms, want_ms) and np.array_equal(bv, want_bv)


def test_unstructured_tables_are_packed_densely():
    """A random table whose motions never share a column in every frame is packed
    four motions a block, not one motion and three pads."""
    rng = np.random.default_rng(2)
    n, m = 9, 200
    dx = rng.integers(-2, 3, (m, n)).astype(np.int32)
    dy = rng.integers(-20, 21, (m, n)).astype(np.int32)
    st = ftb.plan_stats(64, 48, n, dx, dy, 1)
    assert st["pads"] < 4 and st["row_groups"] == 0
