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


def test_golden_is_the_reference():
    if not os.path.exists(REF_DRIVER_SO):
        pytest.skip("reference build absent (make -C oracle ref)")
    from ftoracle import Reference
    R = Reference()
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
