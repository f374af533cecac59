"""The candidate file (write_candidates_csv, io.cpp:82-115) without a GPU: the
writer, built for the host from the product source
(tests/candidates_csv_check.cpp), turns the reference's result fields into the
reference's text byte for byte; its dates equal iso_from_mjd (fits.cpp:474-504)
across day carries, leap years and eras; the track points equal the reference's
ft_get_track_point values. The device search's file is compared
in test_candidates_csv_gpu.py."""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT, golden
from ftoracle import REF_DRIVER_SO

CSRC = os.path.join(ROOT, "fainttrail_b200", "csrc")


def csv_cases():
    """(name, info[5], method, rows (n, 17), flags, the reference's text)."""
    g = golden("candidates_csv_small.npz")
    return [(str(n), g[n + "_info"], str(g[n + "_method"]), g[n + "_rows"], [str(f) for f in g[n + "_flags"]],
             str(g[n + "_csv"])) for n in g["names"]]


@pytest.fixture(scope="module")
def writer(tmp_path_factory):
    gxx = shutil.which("g++")
    if not gxx:
        pytest.skip("no host C++ compiler")
    lib = str(tmp_path_factory.mktemp("csv") / "libcsvcheck.so")
    subprocess.run([gxx, "-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-shared", "-o", lib,
                    os.path.join(ROOT, "tests", "candidates_csv_check.cpp"),
                    os.path.join(CSRC, "candidate_csv.cpp"), "-I" + CSRC], check=True)
    L = C.CDLL(lib)
    f64 = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
    L.ftb_host_candidates_csv.argtypes = [f64, C.c_char_p, f64, C.c_char_p, C.c_int, C.c_char_p, C.c_longlong]
    L.ftb_host_candidates_csv.restype = C.c_longlong
    L.ftb_host_iso_utc.argtypes = [C.c_double, C.c_int, C.c_char_p, C.c_int]
    L.ftb_host_track_points.argtypes = [C.c_double, f64, C.c_int, f64, C.c_int, f64]
    return L


def _text(L, info, method, rows, flags):
    rows = np.ascontiguousarray(np.asarray(rows, np.float64).reshape(-1, 17))
    packed = b"".join(f.encode().ljust(64, b"\0")[:64] for f in flags) or b"\0"
    args = (np.ascontiguousarray(info, np.float64), method.encode(), rows if rows.size else np.zeros(17), packed,
            rows.shape[0])
    size = L.ftb_host_candidates_csv(*args, None, 0)
    buf = C.create_string_buffer(size + 1)
    L.ftb_host_candidates_csv(*args, buf, size + 1)
    return buf.value.decode()


@pytest.mark.parametrize("case", range(2))
def test_writer_matches_reference_text(writer, case):
    name, info, method, rows, flags, want = csv_cases()[case]
    assert _text(writer, info, method, rows, flags) == want, name


def test_fixture_covers_the_columns():
    cases = {c[0]: c for c in csv_cases()}
    null_rows, fixed_flags = cases["null"][3], cases["fixed"][4]
    assert null_rows.shape[0] >= 2 and np.all(null_rows[:, 11] > 0)  # false alarms from the null-tail fit
    assert any("," in f for f in fixed_flags) and any(r[14] == 0 for r in cases["fixed"][3])  # quoted lists, rejects


def test_empty_candidate_list(writer):
    name, info, method, rows, flags, want = csv_cases()[0]
    text = _text(writer, info, method, rows[:0], [])
    assert text == "".join(want.splitlines(keepends=True)[:3])


def test_dates_match_reference(writer):
    if not os.path.exists(REF_DRIVER_SO):
        pytest.skip("reference build absent (make -C oracle ref)")
    from ftoracle import Reference
    R = Reference()
    rng = np.random.default_rng(4)
    mjds = list(rng.uniform(-700000.0, 200000.0, 400)) + [
        61337.90407986, 51544.0, 51543.99999999, 51603.5, 88069.0, 15020.0, 0.0, -0.5, -678941.0, 40587.0,
        40586.9999999999, 59999.999999942, 59999.99999995, 60000.0 - 0.5 / 86400.0 / 100.0]
    buf = C.create_string_buffer(96)
    for mjd in mjds:
        for dec in (0, 1, 2, 3):
            writer.ftb_host_iso_utc(mjd, dec, buf, 96)
            assert buf.value.decode() == R.iso_from_mjd(mjd, dec), (mjd, dec)


@pytest.mark.parametrize("case", range(2))
def test_track_points_match_reference(writer, case):
    g = golden("candidates_csv_small.npz")
    name = csv_cases()[case][0]
    info, rows, t_h, want = g[name + "_info"], g[name + "_rows"], g[name + "_t_h"], g[name + "_tracks"]
    nc, n = rows.shape[0], t_h.size
    assert want.shape == (nc, n, 5) and nc > 0
    out = np.zeros((nc, n, 5))
    writer.ftb_host_track_points(float(info[0]), np.ascontiguousarray(t_h), n, np.ascontiguousarray(rows), nc, out)
    assert np.array_equal(out, want)
