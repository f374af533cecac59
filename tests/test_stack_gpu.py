"""Stack parity on the B200: the CUDA pass through the C ABI against the oracle
(CPU restatement) and the golden vectors from the reference. Bit-exact: equal
max_snr bits (NaN == NaN) and equal best_v everywhere."""
import numpy as np
import pytest

import fainttrail_b200 as ftb
from conftest import golden

pytestmark = pytest.mark.gpu


def same(a, b):
    return np.array_equal(np.asarray(a), np.asarray(b), equal_nan=True)


def run(backend, frames, **kw):
    r = backend.run(ftb.StackPass(frames, **kw))
    return r.max_snr, r.best_v


@pytest.fixture(params=[0, 1, 2, 3, 4, 5, 6, 7, 8],
                ids=["auto", "32x16", "64x8pair", "32x8", "32x4", "32x16shared16w", "32x16shared14w", "32x12",
                     "32x20shared16w"])
def shape(request):
    """Every compiled tile shape (a shape whose windows do not fit falls back)."""
    ftb.set_tile_shape(request.param)
    yield request.param
    ftb.set_tile_shape(0)


@pytest.mark.parametrize("name", ["stack_contract.npz", "stack_constant.npz", "stack_nan_table.npz"])
def test_golden_passes(backend, shape, name):
    g = golden(name)
    ms, bv = run(backend, g["frames"], t_h=g["t_h"], velocities=g["vel"], min_count=int(g["min_count"]))
    assert same(ms, g["max_snr"]) and same(bv, g["best_v"])
    if "dx" in g:
        ms, bv = run(backend, g["frames"], shifts=(g["dx"], g["dy"]), min_count=int(g["min_count"]))
        assert same(ms, g["table_max_snr"]) and same(bv, g["table_best_v"])


def test_tie_known_answer(backend):
    g = golden("stack_constant.npz")
    ms, bv = run(backend, g["frames"], t_h=g["t_h"], velocities=g["vel"], min_count=5)
    assert bv[11, 18] == 0 and abs(ms[11, 18] - np.sqrt(7.0)) < 1e-5


@pytest.mark.parametrize("w,h,n,seed", [(1, 1, 1, 0), (33, 17, 5, 1), (64, 64, 20, 2), (130, 70, 40, 3),
                                        (200, 37, 64, 4), (96, 40, 120, 5), (48, 20, 255, 6)])
def test_random_lattice_passes(backend, oracle, shape, w, h, n, seed):
    rng = np.random.default_rng(seed)
    frames = rng.standard_normal((n, h, w)).astype(np.float32)
    if w * h > 4:
        frames.flat[rng.integers(0, frames.size, 3)] = np.nan
    t = np.sort(rng.uniform(-0.2, 0.2, n))
    span = 0.4
    grid, _ = oracle.velocity_grid(span, 2.0, 60.0, 0.125)
    dx, dy = oracle.shift_table(t, grid)
    mc = oracle.min_count(0.7, n)
    ms, bv = run(backend, frames, t_h=t, velocities=grid, min_count=mc)
    ms2, bv2 = oracle.stack(frames, dx, dy, mc)
    assert same(ms, ms2) and same(bv, bv2)


def test_arbitrary_tables_and_integer_ties(backend, oracle, shape):
    rng = np.random.default_rng(7)
    n, h, w, m = 11, 45, 70, 300
    # small integers: many exact ties between motions
    frames = rng.integers(-3, 4, (n, h, w)).astype(np.float32)
    dx = rng.integers(-30, 31, (m, n)).astype(np.int32)
    dy = rng.integers(-12, 13, (m, n)).astype(np.int32)
    dx[5] += 10000
    dy[9] -= 70000
    for mc in (1, 6, 11):
        ms, bv = run(backend, frames, shifts=(dx, dy), min_count=mc)
        ms2, bv2 = oracle.stack(frames, dx, dy, mc)
        assert same(ms, ms2) and same(bv, bv2), mc


def test_progress_and_cancel(backend, oracle):
    rng = np.random.default_rng(3)
    frames = rng.standard_normal((9, 60, 90)).astype(np.float32)
    t = np.linspace(-0.1, 0.1, 9)
    grid, _ = oracle.velocity_grid(0.2, 5.0, 150.0, 0.125)
    seen = []
    ms, bv = run(backend, frames, t_h=t, velocities=grid, min_count=5)
    r = backend.run(ftb.StackPass(frames, t_h=t, velocities=grid, min_count=5),
                    progress=lambda f, s: seen.append(f) or True)
    assert same(r.max_snr, ms) and same(r.best_v, bv)
    assert seen and seen[-1] == 1.0 and all(b >= a for a, b in zip(seen, seen[1:]))
    with pytest.raises(ftb.Cancelled):
        backend.run(ftb.StackPass(frames, t_h=t, velocities=grid, min_count=5), progress=lambda f, s: f < 0.3)
    # the context stays usable after a cancel
    ms3, bv3 = run(backend, frames, t_h=t, velocities=grid, min_count=5)
    assert same(ms3, ms) and same(bv3, bv)


def test_min_count_above_frame_count(backend, oracle):
    """min_count above the frame count (allowed by validate_pass,
    backend.cpp:89-108): no S/N is defined, so max_snr is 0 and best_v -1
    everywhere, as the reference's CPU backend gives (the pass is not stacked)."""
    g = golden("stack_contract.npz")
    n = g["frames"].shape[0]
    dx, dy = oracle.shift_table(g["t_h"], g["vel"])
    for mc in (n + 1, n + 5):
        ms, bv = run(backend, g["frames"], t_h=g["t_h"], velocities=g["vel"], min_count=mc)
        want = oracle.stack(g["frames"], dx, dy, mc)
        assert same(ms, want[0]) and same(bv, want[1]) and not ms.any() and np.all(bv == -1)
