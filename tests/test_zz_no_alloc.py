"""The allocation-free stacking pass (ft_b200_stack_dev_noalloc).

Some callers cannot allocate device memory during a pass: applications whose
own memory pool owns the GPU and does not let a library grow it, and
latency-bound loops that must not wait on the allocator. For them the pass keeps
its plan tables in a fixed device array inside the library instead of
allocating. This test checks that entry point bit for bit -- the tolerance of
every stacking test here -- against the CPU oracle and against the ordinary
device-resident pass (ft_b200_stack_dev), on two different passes in a row and
on the first pass again (tables left in the shared array by the previous call
must not leak into the next one), on the caller's stream and on the default
stream; a pass whose min_count exceeds its frame count gives the reference's
undefined maps (S/N 0, motion -1). It needs no other test to have run first.
Collected last on purpose: a failure here comes after every other test has run.
"""
import ctypes as C

import numpy as np
import pytest

import fainttrail_b200 as ftb
from ftoracle import Oracle

pytestmark = pytest.mark.gpu


def _bind():
    L = ftb.lib()
    i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
    L.ft_b200_stack_dev_noalloc.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, i32p, i32p, C.c_int,
                                            C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    L.ft_b200_last_error.restype = C.c_char_p
    return L


def _passes(rng, n):
    t = np.sort(rng.uniform(-0.2, 0.2, n))
    g = np.arange(-12, 13) * 3.0
    vel = np.array([(vx, vy) for vy in g for vx in g if 6.0 <= np.hypot(vx, vy) <= 36.0])
    r = lambda v: (np.sign(v) * np.floor(np.abs(v) + 0.5)).astype(np.int32)  # half away from zero
    lattice = (r(vel[:, :1] * t[None, :]), r(vel[:, 1:] * t[None, :]), 14)
    m = 333
    table = (rng.integers(-9, 10, (m, n)).astype(np.int32), rng.integers(-7, 8, (m, n)).astype(np.int32), 3)
    table[0][17] += 5000  # a motion whose frames never cover
    return [lattice, table]


def test_no_alloc_pass_matches_oracle_and_stack_dev_twice():
    import torch
    L = _bind()
    O = Oracle()
    dev = ftb.Device(0)
    rng = np.random.default_rng(11)
    n, h, w = 20, 150, 200
    host = rng.standard_normal((n, h, w)).astype(np.float32)
    host[3, 10, 20] = np.nan
    frames = torch.from_numpy(host).cuda()
    stream = torch.cuda.current_stream().cuda_stream
    passes = _passes(rng, n)
    for k, (dx, dy, mc) in enumerate(passes + passes[:1] + passes[1:]):
        oracle_ms, oracle_bv = O.stack(host, dx, dy, mc)
        want_ms = torch.empty((h, w), device="cuda")
        want_bv = torch.empty((h, w), dtype=torch.int32, device="cuda")
        dev.stack_dev(frames.data_ptr(), w, h, w, n, dx, dy, mc, want_ms.data_ptr(), want_bv.data_ptr())
        got_ms = torch.full((h, w), -7.0, device="cuda")
        got_bv = torch.full((h, w), -7, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        # the last call goes to the default stream (NULL)
        rc = L.ft_b200_stack_dev_noalloc(frames.data_ptr(), w, h, w, n, dx, dy, dx.shape[0], mc, got_ms.data_ptr(),
                                         got_bv.data_ptr(), stream if k < 3 else None)
        assert rc == ftb.FT_B200_OK, L.ft_b200_last_error(None)
        got_ms, got_bv = got_ms.cpu().numpy(), got_bv.cpu().numpy()
        assert np.array_equal(got_bv, oracle_bv)
        assert np.array_equal(got_ms, oracle_ms, equal_nan=True)
        assert np.array_equal(got_bv, want_bv.cpu().numpy())
        assert np.array_equal(got_ms, want_ms.cpu().numpy(), equal_nan=True)
    dev.close()


def test_no_alloc_min_count_above_frame_count():
    import torch
    L = _bind()
    O = Oracle()
    rng = np.random.default_rng(5)
    n, h, w = 6, 40, 72  # a row pitch of 288 bytes: a multiple of 16
    host = rng.standard_normal((n, h, w)).astype(np.float32)
    frames = torch.from_numpy(host).cuda()
    dx = rng.integers(-3, 4, (9, n)).astype(np.int32)
    dy = rng.integers(-3, 4, (9, n)).astype(np.int32)
    oracle_ms, oracle_bv = O.stack(host, dx, dy, n + 1)
    got_ms = torch.full((h, w), -7.0, device="cuda")
    got_bv = torch.full((h, w), -7, dtype=torch.int32, device="cuda")
    rc = L.ft_b200_stack_dev_noalloc(frames.data_ptr(), w, h, w, n, dx, dy, 9, n + 1, got_ms.data_ptr(),
                                     got_bv.data_ptr(), None)
    assert rc == ftb.FT_B200_OK, L.ft_b200_last_error(None)
    got_ms, got_bv = got_ms.cpu().numpy(), got_bv.cpu().numpy()
    assert np.array_equal(got_ms, oracle_ms) and np.array_equal(got_bv, oracle_bv)
    assert not np.signbit(got_ms).any() and (got_ms == 0).all() and (got_bv == -1).all()


def test_no_alloc_refuses_oversized_plans():
    import torch
    L = _bind()
    n, h, w, m = 60, 8, 32, 120000  # 7.2 million (motion, frame) pairs: beyond the fixed tables
    frames = torch.zeros((n, h, w), device="cuda")
    out = torch.empty((h, w), device="cuda")
    bv = torch.empty((h, w), dtype=torch.int32, device="cuda")
    dx = np.zeros((m, n), np.int32)
    rc = L.ft_b200_stack_dev_noalloc(frames.data_ptr(), w, h, w, n, dx, dx, m, 3, out.data_ptr(), bv.data_ptr(),
                                     None)
    assert rc == ftb.FT_B200_ERROR
    assert b"at most 32 MiB" in L.ft_b200_last_error(None)
