"""The registration check on the device (ft_b200_check_registration and _dev)
and inside a search (align): bit-identical to the reference's
check_registration (registration.cpp:260-312) on the golden cases and on
rendered star fields (drift, rotation, scale, meridian flip, tied peaks, NaN
blanks, tied and unsorted times, a frame large enough to sample every other
pixel); a search with align "check" refuses frames that are not registered with
the reference's message (preprocess.cpp:618-619) and otherwise equals the same
search without the check."""
import numpy as np
import pytest

from test_registration import golden_cases

pytestmark = pytest.mark.gpu


def _render(w, h, stars, T, rng, integer):
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    img = 100.0 + rng.normal(0, 3.0, (h, w))
    a, b, tx, ty = T
    for x, y, f in stars:
        u, v = a * x - b * y + tx, b * x + a * y + ty
        if -10 < u < w + 10 and -10 < v < h + 10:
            x0, x1, y0, y1 = max(0, int(u) - 8), min(w, int(u) + 9), max(0, int(v) - 8), min(h, int(v) + 9)
            img[y0:y1, x0:x1] += f * np.exp(-((xx[y0:y1, x0:x1] - u) ** 2 + (yy[y0:y1, x0:x1] - v) ** 2) / 2.88)
    return (np.round(img) if integer else img).astype(np.float32)


def field(seed, w=256, h=200, n=12, nstars=80, drift=(0.0, 0.0), rot_deg=0.0, scale=1.0, flip_after=None,
          integer=False, saturate=False, blanks=0, times=None):
    """A star field seen n times: frame i maps the sky by a similarity that grows
    with time (rotation, scale) plus a drift of i * drift px, optionally turned
    by 180 degrees from frame flip_after on. Returns (frames, t_h)."""
    rng = np.random.default_rng(seed)
    stars = [(rng.uniform(0, w), rng.uniform(0, h), 60000.0 if saturate else rng.uniform(30, 3000))
             for _ in range(nstars)]
    t = np.arange(n, dtype=np.float64) * 0.05 if times is None else np.asarray(times, np.float64)
    cx, cy = 0.5 * (w - 1), 0.5 * (h - 1)
    frames = []
    for i in range(n):
        k = t[i] / max(t.max(), 1e-9)
        th, s = np.deg2rad(rot_deg * k), 1 + (scale - 1) * k
        a, b = s * np.cos(th), s * np.sin(th)
        tx, ty = cx - (a * cx - b * cy) + drift[0] * i, cy - (b * cx + a * cy) + drift[1] * i
        if flip_after is not None and i >= flip_after:
            a, b, tx, ty = -a, -b, 2 * cx - tx + 0.3, 2 * cy - ty - 0.2
        img = _render(w, h, stars, (a, b, tx, ty), rng, integer)
        if saturate:
            img = np.minimum(img, 4000.0)
        for _ in range(blanks):
            x0, y0 = rng.integers(0, w - 5), rng.integers(0, h - 5)
            img[y0:y0 + rng.integers(1, 5), x0:x0 + rng.integers(1, 5)] = np.nan
        frames.append(img)
    return np.ascontiguousarray(np.stack(frames)), t


FIELDS = {
    "registered": dict(seed=1),
    "drift": dict(seed=2, drift=(0.4, -0.25)),
    "slow drift": dict(seed=3, drift=(0.1, 0.1)),
    "rotation": dict(seed=4, rot_deg=0.8, drift=(0.05, 0.0)),
    "scale": dict(seed=5, scale=1.004),
    "flip": dict(seed=6, flip_after=6),
    "few stars": dict(seed=7, nstars=4),
    "11 stars": dict(seed=8, nstars=11, drift=(0.3, 0.0)),
    "integer": dict(seed=9, integer=True, drift=(0.2, 0.3)),
    "saturated ties": dict(seed=10, saturate=True, integer=True, drift=(0.3, 0.0)),
    "blanks": dict(seed=11, blanks=60, drift=(0.25, 0.0)),
    "time ties": dict(seed=12, times=[0, .1, .1, .1, .2, .2, .3, .3, .3, .3, .4, .4], drift=(0.3, 0.2)),
    "unsorted": dict(seed=13, times=[.3, 0, .5, .1, .45, .2, .05, .6, .35, .25, .55, .15], drift=(0.2, 0.0)),
    "two frames": dict(seed=14, n=2),
    "big shift": dict(seed=15, drift=(6.0, -4.0), nstars=150),
    "dense": dict(seed=16, nstars=600, drift=(0.15, 0.0)),
    "tiny": dict(seed=17, w=30, h=24, nstars=10),
    "thin": dict(seed=18, w=400, h=12, nstars=40),
    "odd sizes": dict(seed=19, n=17, w=181, h=163, drift=(0.12, -0.09)),
    "40 frames": dict(seed=20, n=40, drift=(0.05, 0.04), nstars=120),
    "large": dict(seed=40, w=1200, h=900, n=3, nstars=500, drift=(0.9, 0.3)),
}


@pytest.mark.parametrize("case", range(5))
def test_golden_cases(device, case):
    name, frames, t, want = golden_cases()[case]
    assert device.check_registration(frames, t) == want, name


@pytest.mark.parametrize("name", list(FIELDS))
def test_rendered_fields_match_reference(device, reference, name):
    frames, t = field(**FIELDS[name])
    assert device.check_registration(frames, t) == reference.check_registration(frames, t)


def test_device_frames_with_row_pitch(device, reference):
    import torch
    frames, t = field(**FIELDS["drift"])
    n, h, w = frames.shape
    pitch = w + 13
    buf = torch.zeros((n, h, pitch), dtype=torch.float32, device="cuda")
    buf[:, :, :w] = torch.from_numpy(frames).cuda()
    torch.cuda.synchronize()
    got = device.check_registration_dev(buf.data_ptr(), w, h, pitch, n, t)
    assert got == reference.check_registration(frames, t)


def _sequence(name):
    frames, t = field(**FIELDS[name])
    mjd = 60000.0 + t / 24.0
    return frames, mjd, np.full(t.size, 30.0)


def test_search_refuses_unregistered_frames(device, reference):
    frames, mjd, exp = _sequence("drift")
    want = reference.check_registration(frames, (mjd - mjd[0]) * 24.0)
    assert want["registered"] == 0
    with pytest.raises(RuntimeError) as e:
        device.search(frames, mjd, exp, fwhm_px=2.0, null_runs=1, align="check")
    assert want["message"] in str(e.value)
    with pytest.raises(RuntimeError, match="does not align frames"):
        device.search(frames, mjd, exp, fwhm_px=2.0, null_runs=1, align="auto")


def test_search_with_check_equals_search_without(device, reference):
    """Registered frames given in shuffled order: the search sorts them by time,
    checks the sorted sequence as the reference does, and returns what the
    search without the check returns, plus the check."""
    frames, mjd, exp = _sequence("registered")
    perm = np.random.default_rng(3).permutation(mjd.size)
    kw = dict(fwhm_px=2.0, null_runs=1)
    plain = device.search(frames[perm], mjd[perm], exp[perm], **kw)
    checked = device.search(frames[perm], mjd[perm], exp[perm], align="check", **kw)
    assert checked["registration"] == reference.check_registration(frames, (mjd - mjd[0]) * 24.0)
    assert checked["registration"]["measured"] == 1 and checked["registration"]["registered"] == 1
    assert plain["registration"]["measured"] == 0 and plain["registration"]["registered"] == 1
    assert checked["threshold"] == plain["threshold"] and checked["peaks"] == plain["peaks"]
    assert np.array_equal(checked["max_snr"], plain["max_snr"], equal_nan=True)
    assert np.array_equal(checked["best_v"], plain["best_v"])
