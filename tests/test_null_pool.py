"""The null-run pooling shortcut on the host (ft_b200_pool_null_peaks): the
search pools a null run's peaks without the full std::sort of order_peaks
(search.cpp:132), because equal S/N values are interchangeable in the pooled
list and only the set of peaks screened for artefacts depends on how ties are
ordered. These cases check the shortcut against the reference's full sort --
the same libstdc++ std::sort on the same raster-ordered input -- including
heavy ties, ties straddling the screening boundary, the truncation, and no
screening at all."""
import ctypes as C

import numpy as np
import pytest

import fainttrail_b200 as ftb


def pool(peaks, flags, keep, tested, mode):
    L = ftb.lib()
    L.ft_b200_pool_null_peaks.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p,
                                          C.c_int]
    arr = (ftb.Peak * max(1, len(peaks)))(*[ftb.Peak(*p) for p in peaks])
    fl = np.ascontiguousarray(flags, dtype=np.uint8)
    out = np.empty(max(1, len(peaks)), np.float32)
    n = L.ft_b200_pool_null_peaks(arr, len(peaks), fl.ctypes.data_as(C.c_void_p), keep, tested, mode,
                                  out.ctypes.data_as(C.c_void_p), out.size)
    assert n >= 0
    return out[:n].copy()


@pytest.mark.parametrize("count,levels,keep,tested,seed", [
    (0, 10, 20000, 3000, 0), (50, 1000, 20000, 3000, 1), (5000, 40, 20000, 3000, 2), (5000, 100000, 20000, 3000, 3),
    (30000, 300, 20000, 3000, 4), (30000, 1000000, 20000, 3000, 5), (4000, 7, 20000, 3000, 6), (5000, 50, 2000, 3000, 7),
    (8000, 25, 20000, 0, 8), (3001, 2, 20000, 3000, 9), (3000, 5, 20000, 3000, 10)])
def test_shortcut_equals_full_sort(count, levels, keep, tested, seed):
    rng = np.random.default_rng(seed)
    # raster order: distinct pixels, S/N from `levels` distinct values (ties)
    pix = rng.choice(200000, size=count, replace=False)
    pix.sort()
    snr = (3.0 + rng.integers(0, levels, count) / levels * 5.0).astype(np.float32)
    peaks = [(int(p % 500), int(p // 500), float(s), int(rng.integers(0, 100))) for p, s in zip(pix, snr)]
    flags = rng.random(count) < 0.3
    a = pool(peaks, flags, keep, tested, 0)
    b = pool(peaks, flags, keep, tested, 1)
    assert a.shape == b.shape and np.array_equal(a, b)
