"""The C-ABI library loads and exports every entry point include/ft_b200.h
declares; host-side argument checks. No GPU needed."""
import ctypes as C
import os

import numpy as np
import pytest

import fainttrail_b200 as ftb
from conftest import ROOT


def test_library_exports_every_declared_symbol():
    L = ftb.lib()
    names = ftb.exported_symbols()
    assert "ft_b200_stack" in names and "ft_b200_open" in names
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_open_without_gpu_reports_an_error():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    assert ftb.lib().ft_b200_open(0, 0.0, C.byref(h)) == ftb.FT_B200_ERROR
    assert ftb.lib().ft_b200_last_error(None)


def test_null_context_is_an_error():
    L = ftb.lib()
    f = np.zeros((1, 4, 4), np.float32)
    d = np.zeros((1, 1), np.int32)
    out = np.zeros((4, 4), np.float32)
    bv = np.zeros((4, 4), np.int32)
    assert L.ft_b200_stack(None, f, 4, 4, 1, d, d, 1, 1, out, bv, ftb.PROGRESS_FN(), None) == ftb.FT_B200_ERROR


def test_validate_pass_mirrors_reference():
    f = np.zeros((3, 5, 6), np.float32)
    with pytest.raises(RuntimeError, match="missing times"):
        ftb.validate_pass(ftb.StackPass(f, min_count=1))
    with pytest.raises(RuntimeError, match="frame and time counts"):
        ftb.validate_pass(ftb.StackPass(f, t_h=[0.0, 1.0], velocities=[(1.0, 0.0)]))
    with pytest.raises(RuntimeError, match="shift table and frame counts"):
        ftb.validate_pass(ftb.StackPass(f, shifts=(np.zeros((4, 2)), np.zeros((4, 2)))))
    with pytest.raises(RuntimeError, match="min_count"):
        ftb.validate_pass(ftb.StackPass(f, t_h=[0, 1, 2], velocities=[(1.0, 0.0)], min_count=0))
    ftb.validate_pass(ftb.StackPass(f, t_h=[0, 1, 2], velocities=[(1.0, 0.0)]))
    with pytest.raises(RuntimeError, match="unknown or unavailable"):
        ftb.make_backend("cuda")


def test_host_only_entries_without_a_gpu():
    """Entries that do no device work answer on a machine without a GPU: tile
    shape selection and its checks, the tuner's (empty) cache, and the argument
    checks of the null-threshold and pooling entries."""
    import ctypes as C

    import fainttrail_b200 as ftb
    L = ftb.lib()
    assert ftb.tile_shape() == 0
    for shape in range(0, 9):
        ftb.set_tile_shape(shape)
        assert ftb.tile_shape() == shape
    ftb.set_tile_shape(0)
    for bad in (-1, 9, 99):
        with pytest.raises(ValueError, match="tile shape"):
            ftb.set_tile_shape(bad)
    assert ftb.tile_shape() == 0
    ftb.clear_tuned_shapes()
    assert ftb.tuned_shapes() == {}
    with pytest.raises(RuntimeError, match="bad sizes"):
        ftb.null_threshold([5.0, 4.0], 1, 2.5, 0, 10, 100)
    L.ft_b200_pool_null_peaks.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p,
                                          C.c_int]
    assert L.ft_b200_pool_null_peaks(None, 3, None, 20000, 3000, 0, None, 0) == -1


def test_registration_entries_check_their_arguments():
    """The registration entries refuse a missing context or result, and the
    drift-check struct has the C layout (4 ints, 5 doubles, a 1024-byte message)."""
    import ctypes as C

    import fainttrail_b200 as ftb
    L = ftb.lib()
    out = ftb.DriftCheck()
    assert C.sizeof(ftb.DriftCheck) == 4 * 4 + 5 * 8 + 1024
    f = np.zeros((3, 16, 16), np.float32)
    t = np.arange(3, dtype=np.float64)
    assert L.ft_b200_check_registration(None, f, 16, 16, 3, t, C.byref(out)) == ftb.FT_B200_ERROR
    assert L.ft_b200_check_registration_dev(None, None, 16, 16, 16, 3, t, C.byref(out)) == ftb.FT_B200_ERROR
    assert L.ft_b200_result_registration(None, C.byref(out)) == ftb.FT_B200_ERROR


def test_only_the_declared_entries_have_c_names():
    """Internal helpers of the C ABI layer keep internal linkage: every exported
    unmangled symbol is one of the ft_b200_ entries the header declares."""
    import shutil
    import subprocess

    nm = shutil.which("nm")
    if not nm:
        pytest.skip("no nm")
    out = subprocess.run([nm, "-D", "--defined-only", ftb.LIB_PATH], capture_output=True, text=True, check=True)
    names = [line.split()[-1] for line in out.stdout.splitlines() if line.split()[1] in ("T", "D", "B")]
    c_names = {n for n in names if not n.startswith("_Z")}
    assert c_names <= set(ftb.exported_symbols()), sorted(c_names - set(ftb.exported_symbols()))


def test_candidate_record_layout_and_checks():
    """ft_b200_candidate has ft_candidate's layout (2 ints, 18 doubles, 64 flag
    bytes); the candidate and track-point getters refuse a missing result."""
    import ctypes as C

    import fainttrail_b200 as ftb
    assert C.sizeof(ftb.CandidateRecord) == 2 * 4 + 18 * 8 + 64
    L = ftb.lib()
    rec = ftb.CandidateRecord()
    assert L.ft_b200_result_candidate(None, 0, C.byref(rec)) == ftb.FT_B200_ERROR
    d = C.c_double()
    assert L.ft_b200_result_track_point(None, 0, 0, *[C.byref(d)] * 5) == ftb.FT_B200_ERROR


def test_unknown_parameters_are_errors():
    """A misspelt search or stage parameter is refused, not silently ignored."""
    import fainttrail_b200 as ftb
    L = ftb.lib()
    with pytest.raises(TypeError, match="nul_runs"):
        ftb.Device._search_params(L, {"nul_runs": 3})
    p = ftb.Device._search_params(L, {"null_runs": 5, "calibrated_tail": (1.0, 2.0, 3.0, 4.0), "align": "check"})
    assert p.null_runs == 5 and list(p.calibrated_tail) == [1.0, 2.0, 3.0, 4.0] and p.align == 1
    with pytest.raises(TypeError, match="clip"):
        ftb._set_fields(ftb.StageParams(), {"clip": 3.0}, "stage")


C_PROGRAM = r"""
#include <stdio.h>
#include "ft_b200.h"
int main(void) {
    ft_b200_search_params q;
    ft_b200_stage_params s;
    ft_b200_ctx* ctx = 0;
    ft_b200_search_params_default(&q);
    ft_b200_stage_params_default(&s);
    printf("%s %d %g %d %g %d\n", ft_b200_version(), q.null_runs, q.vmax_pxh, q.align, s.clip_sigma,
           ft_b200_open(0, 0.0, &ctx) == FT_B200_OK);
    if (ctx) ft_b200_close(ctx);
    return 0;
}
"""


def test_header_is_plain_c(tmp_path):
    """include/ft_b200.h compiles as strict C99 and a C program links against
    the library and calls its host-side entries (no GPU work)."""
    import shutil
    import subprocess

    gcc = shutil.which("gcc")
    if not gcc:
        pytest.skip("no C compiler")
    src = tmp_path / "abi.c"
    src.write_text(C_PROGRAM)
    exe = tmp_path / "abi"
    lib_dir = os.path.dirname(ftb.LIB_PATH)
    subprocess.run([gcc, "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", "-I" + os.path.join(ROOT, "include"),
                    str(src), "-L" + lib_dir, "-lft_b200", "-Wl,-rpath," + lib_dir, "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    assert out[0].startswith("0.9.1") and out[1:5] == ["3", "40", "0", "8"]
