"""Preprocessing stage parity on the B200: ft_b200_stage against the oracle's
build_stage restatement and the reference's own outputs (golden vectors).
Bit-exact: filtered frames, static sky, mask, per-frame sigma, cosmic-ray counts."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu
KEYS = ("filtered", "static_sky", "mask", "sigma", "cr")


def same(a, b):
    return np.array_equal(np.asarray(a), np.asarray(b), equal_nan=True)


def check(got, want):
    for k in KEYS:
        assert same(got[k], want[k]), k


def test_golden_stage(device):
    g = golden("stage_small.npz")
    got = device.stage(g["sub"], g["t_h"], float(g["fwhm"]))
    check(got, g)


def test_null_time_orders(device, oracle):
    g = golden("stage_small.npz")
    orders = oracle.null_orders(g["t_h"], 3, 12345)
    for t in orders:
        check(device.stage(g["sub"], t, float(g["fwhm"])), oracle.build_stage(g["sub"], t, float(g["fwhm"])))


@pytest.mark.parametrize("n,w,h,seed,fwhm", [(5, 40, 30, 1, 2.5), (20, 97, 61, 2, 2.5), (40, 128, 96, 3, 3.3),
                                             (64, 70, 50, 4, 2.0), (120, 48, 40, 5, 4.0), (200, 40, 24, 6, 2.5),
                                             (12, 90, 70, 7, 7.0), (16, 150, 100, 8, 1.2)])
def test_random_sequences(device, oracle, n, w, h, seed, fwhm):
    rng = np.random.default_rng(seed)
    sub = rng.normal(0, 10, (n, h, w)).astype(np.float32)
    # stars (static), a few cosmic rays, blank borders, integer-valued ties
    for _ in range(6):
        x, y = rng.integers(3, w - 3), rng.integers(3, h - 3)
        sub[:, y - 1:y + 2, x - 1:x + 2] += 400.0
    for i in range(n):
        x, y = rng.integers(2, w - 2), rng.integers(2, h - 2)
        sub[i, y, x] += 900.0
    sub[:, :, :3] = np.nan
    sub[rng.integers(0, n), 5:9, 10:14] = np.nan
    sub[: n // 3, -2:, :] = np.nan
    sub[: n // 2, 2:4, 20:24] = np.nan  # fewer finite values than the static sky needs
    sub[:, 7, :] = np.round(sub[:, 7, :])
    t = np.sort(rng.uniform(-0.3, 0.3, n))
    rng.shuffle(t)
    check(device.stage(sub, t, fwhm), oracle.build_stage(sub, t, fwhm))


def test_parameters(device, oracle):
    g = golden("stage_small.npz")
    for kw in (dict(static_exclude=0), dict(static_exclude=3), dict(clip_sigma=3.0, cr_sigma=4.0),
               dict(mask_scatter=1.8, weight_scatter=1.2)):
        check(device.stage(g["sub"], g["t_h"], 2.5, **kw), oracle.build_stage(g["sub"], g["t_h"], 2.5, **kw))


def test_stage_then_stack_matches_reference_pass(device, backend, oracle):
    import fainttrail_b200 as ftb
    g = golden("stage_small.npz")
    st = device.stage(g["sub"], g["t_h"], float(g["fwhm"]))
    grid, _ = oracle.velocity_grid(float(g["span_h"]), 4.0, 40.0, 0.5)
    mc = oracle.min_count(0.7, len(g["t_h"]))
    r = backend.run(ftb.StackPass(st["filtered"], t_h=g["t_h"], velocities=grid, min_count=mc))
    dx, dy = oracle.shift_table(g["t_h"], grid)
    ms, bv = oracle.stack(g["filtered"], dx, dy, mc)
    assert same(r.max_snr, ms) and same(r.best_v, bv)


def test_noise_normalisation(device, reference):
    """The reference's test_noise_normalisation (tests/test_main.cpp:146-167) on
    the device stage: on a star field without movers (192 x 192 x 40, hot pixels,
    cosmic rays), every seventh filtered frame has mean |m| < 0.1 and standard
    deviation in (0.9, 1.15) over the unmasked pixels 10 px inside the edge."""
    R = reference
    frames, mjd, exp = R.simulate(width=192, height=192, nframes=40, exptime_s=45.0, cadence_s=60.0, nstars=200,
                                  hot_pixels=15, cosmic_rays_per_frame=2.0, nmovers=0, seed=11)
    prep = R.prepare(frames, mjd, exp, vmin_pxh=8.0, vmax_pxh=30.0, null_runs=2)
    got = device.stage(prep.images()["sub"], prep.vectors()["t_h"], prep.fwhm)
    flt, mask = got["filtered"], got["mask"]
    inner = np.zeros(mask.shape, bool)
    inner[10:-10, 10:-10] = True
    keep = inner & (mask != 0.0)
    for i in range(0, flt.shape[0], 7):
        v = flt[i][keep].astype(np.float64)
        mean, sd = v.mean(), v.std()
        assert abs(mean) < 0.1 and 0.9 < sd < 1.15


def test_device_frames_with_row_pitch(device):
    """ft_b200_stage_dev on frames in HBM with an odd row pitch: the golden
    outputs, written into the caller's layout; NULL outputs are skipped."""
    import torch
    g = golden("stage_small.npz")
    sub = np.ascontiguousarray(g["sub"], np.float32)
    n, h, w = sub.shape
    pitch = w + 5
    d_sub = torch.full((n, h, pitch), 7.0, dtype=torch.float32, device="cuda")
    d_sub[:, :, :w] = torch.from_numpy(sub).cuda()
    d_filt = torch.full((n, h, pitch), -3.0, dtype=torch.float32, device="cuda")
    d_sky = torch.full((h, pitch), -3.0, dtype=torch.float32, device="cuda")
    d_mask = torch.full((h, pitch), -3.0, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    got = device.stage_dev(d_sub.data_ptr(), w, h, pitch, n, g["t_h"], float(g["fwhm"]), d_filt.data_ptr(),
                           d_sky.data_ptr(), d_mask.data_ptr())
    got.update(filtered=d_filt[:, :, :w].cpu().numpy(), static_sky=d_sky[:, :w].cpu().numpy(),
               mask=d_mask[:, :w].cpu().numpy())
    check(got, g)
    assert torch.all(d_filt[:, :, w:] == -3.0) and torch.all(d_sky[:, w:] == -3.0)  # padding untouched
    only = device.stage_dev(d_sub.data_ptr(), w, h, pitch, n, g["t_h"], float(g["fwhm"]))
    assert same(only["sigma"], g["sigma"]) and same(only["cr"], g["cr"])


def bits_equal(a, b):
    """Bit for bit, the sign of zero included; NaN where the other is NaN."""
    a, b = np.asarray(a, np.float32), np.asarray(b, np.float32)
    na, nb = np.isnan(a), np.isnan(b)
    return np.array_equal(na, nb) and np.array_equal(a.view(np.uint32)[~na], b.view(np.uint32)[~nb])


@pytest.mark.parametrize("n,seed", [(9, 1), (20, 2), (31, 3), (40, 4), (64, 5), (65, 6), (100, 7), (129, 8)])
def test_ties_and_signed_zeros(device, oracle, n, seed):
    """Small integer values with +0.0 and -0.0 among them: most sorted positions
    are ties, resolved by time rank as the reference's sort of (value, rank)
    pairs does, and the leave-out medians' middle pairs are often zeros of both
    signs. Static sky and filtered frames must match the oracle bit for bit."""
    rng = np.random.default_rng(seed)
    h, w = 24, 70
    sub = rng.integers(-2, 3, (n, h, w)).astype(np.float32)
    zeros = sub == 0
    sub[zeros & (rng.random(sub.shape) < 0.5)] = -0.0
    sub[:, :, :2] = np.nan
    sub[rng.integers(0, n), 3:6, 10:20] = np.inf
    t = np.sort(rng.uniform(-0.3, 0.3, n))
    rng.shuffle(t)
    got = device.stage(sub, t, 2.5)
    want = oracle.build_stage(sub, t, 2.5)
    assert bits_equal(got["static_sky"], want["static_sky"])
    assert bits_equal(got["filtered"], want["filtered"])
    assert same(got["sigma"], want["sigma"]) and same(got["mask"], want["mask"])
