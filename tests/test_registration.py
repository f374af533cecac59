"""The registration check (check_registration, registration.cpp:260-312) without
a GPU: its host half and per-pixel star test, built for the host from the
product sources (tests/registration_host_check.cpp), reproduce the reference's
golden verdicts; the golden verdicts are the reference's own where it is built;
the Python side maps the align modes. The device scan is checked against the
reference in test_registration_gpu.py."""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT, golden
from ftoracle import REF_DRIVER_SO, drift_dict

CSRC = os.path.join(ROOT, "fainttrail_b200", "csrc")


def golden_cases():
    """(name, frames (3, h, w) with NaN blanks, t_h, the reference's verdict)."""
    g = golden("registration_small.npz")
    out = []
    for name in g["names"]:
        name = str(name)
        fr = g[name + "_frames"].astype(np.float32)
        nan = np.unpackbits(g[name + "_nan"], count=fr.size).reshape(fr.shape).astype(bool)
        fr[nan] = np.nan
        out.append((name, fr, g[name + "_t"], drift_dict(g[name + "_values"], str(g[name + "_message"]))))
    return out


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


@pytest.fixture(scope="module")
def host_check(tmp_path_factory):
    gxx = shutil.which("g++")
    if not gxx:
        pytest.skip("no host C++ compiler")
    lib = str(tmp_path_factory.mktemp("registration") / "libregcheck.so")
    subprocess.run([gxx, "-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-shared", "-o", lib,
                    os.path.join(ROOT, "tests", "registration_host_check.cpp"),
                    os.path.join(CSRC, "registration_host.cpp"), "-I" + CSRC], check=True)
    L = C.CDLL(lib)
    f32 = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
    f64 = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
    L.ftb_host_check_registration.argtypes = [f32, C.c_int, C.c_int, C.c_int, f64, f64, C.c_char_p, C.c_int]

    def run(frames, t_h):
        frames = np.ascontiguousarray(frames, np.float32)
        n, h, w = frames.shape
        out = np.zeros(9)
        msg = C.create_string_buffer(1024)
        L.ftb_host_check_registration(frames, n, w, h, np.ascontiguousarray(t_h, np.float64), out, msg, 1024)
        return drift_dict(out, msg.value.decode())
    return run


def test_golden_cases_cover_the_verdicts():
    cases = {name: want for name, _, _, want in golden_cases()}
    assert cases["registered"]["measured"] == 1 and cases["registered"]["registered"] == 1
    assert cases["drift"]["registered"] == 0 and "not registered" in cases["drift"]["message"]
    assert "rotation 180.0 deg" in cases["flip"]["message"]
    assert cases["few"]["measured"] == 0 and cases["few"]["registered"] == 1


@pytest.mark.parametrize("case", range(5))
def test_host_half_matches_golden(host_check, case):
    name, frames, t, want = golden_cases()[case]
    assert host_check(frames, t) == want, name


def test_frame_choice_follows_time_not_position(host_check):
    """The first, middle and last frame are chosen by time: the same frames in
    another order give the same verdict."""
    name, frames, t, want = golden_cases()[1]
    perm = [2, 0, 1]
    assert host_check(frames[perm], t[perm]) == want


def test_fewer_than_three_frames_are_not_measured(host_check):
    _, frames, t, _ = golden_cases()[1]
    got = host_check(frames[:2], t[:2])
    assert got["measured"] == 0 and got["registered"] == 1 and got["message"] == ""


def _reference():
    if not os.path.exists(REF_DRIVER_SO):
        pytest.skip("reference build absent (make -C oracle ref)")
    from ftoracle import Reference
    return Reference()


@pytest.mark.parametrize("name", list(FIELDS))
def test_host_half_matches_reference_on_rendered_fields(host_check, name):
    frames, t = field(**FIELDS[name])
    assert host_check(frames, t) == _reference().check_registration(frames, t)


def test_tied_times_beyond_sixteen_frames(host_check):
    """40 frames drifting by whole pixels with only 6 distinct times, given in a
    shuffled order: which of the tied frames count as first, middle and last is
    decided by the reference's std::sort of the frame indices (introsort beyond
    16 elements), and the verdict shows it."""
    frames, _ = field(seed=21, w=160, h=128, n=40, nstars=150, drift=(0.35, -0.2))
    t = np.floor(np.arange(40) / 7.0) * 0.1
    perm = np.random.default_rng(8).permutation(40)
    frames, t = np.ascontiguousarray(frames[perm]), t[perm]
    want = _reference().check_registration(frames, t)
    assert want["measured"] == 1
    assert host_check(frames, t) == want


def test_golden_is_the_reference():
    R = _reference()
    for name, frames, t, want in golden_cases():
        assert R.check_registration(frames, t) == want, name


def test_align_modes():
    import fainttrail_b200 as ftb
    L = ftb.lib()
    assert ftb.Device._search_params(L, {}).align == 0
    assert ftb.Device._search_params(L, {"align": "check"}).align == 1
    assert ftb.Device._search_params(L, {"align": "auto"}).align == 2
    with pytest.raises(ValueError, match="resample"):
        ftb.Device._search_params(L, {"align": "always"})
