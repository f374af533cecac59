"""FaintTrail B200 search backend: Python host binding over the C ABI.

The public C ABI is include/ft_b200.h, implemented by the in-tree CUDA library
fainttrail_b200/libft_b200.so (built by fainttrail_b200/build.py). This module
mirrors the reference's plugin interface for the stacking pass
(FaintTrail include/fainttrail/backend.hpp:71-139): ``StackPass``,
``StackResult``, ``SearchBackend.run``, ``make_backend``, ``validate_pass``.
There is no CPU fallback: importing the binding without the built library, or
running it without a B200, raises.
"""
import ctypes as C
import os
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libft_b200.so")

FT_B200_OK, FT_B200_ERROR, FT_B200_CANCELLED = 0, 1, 2

_lib = None
_lock = threading.Lock()

PROGRESS_FN = C.CFUNCTYPE(C.c_int, C.c_double, C.c_char_p, C.c_void_p)

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


class StageParams(C.Structure):
    """ft_b200_stage_params: the stage's SearchParams fields (search.hpp:18-90)."""
    _fields_ = [("fwhm_px", C.c_double), ("static_exclude", C.c_int), ("clip_sigma", C.c_double),
                ("cr_sigma", C.c_double), ("mask_scatter", C.c_double), ("weight_scatter", C.c_double)]


class SearchParams(C.Structure):
    """ft_b200_search_params: ft_params (fainttrail.h:32-54) + null-model fields."""
    _fields_ = [(n, C.c_double) for n in (
        "vmin_pxh", "vmax_pxh", "grid_tol_px", "fwhm_px", "clip_sigma", "cr_sigma", "mask_scatter",
        "weight_scatter", "min_coverage", "threshold_snr", "min_snr_floor", "target_false_per_run",
        "max_frame_fraction", "half_tolerance")] + [
        ("static_exclude", C.c_int), ("null_runs", C.c_int), ("max_candidates", C.c_int), ("edge_px", C.c_int),
        ("threads", C.c_int), ("seed", C.c_ulonglong), ("null_tested", C.c_int), ("null_model_gauss", C.c_int),
        ("passes_per_launch", C.c_int), ("shard_index", C.c_int), ("shard_count", C.c_int),
        ("calibrated_threshold", C.c_double), ("calibrated_tail", C.c_double * 4), ("align", C.c_int),
        ("reg_dx", C.c_void_p), ("reg_dy", C.c_void_p)]


ALIGN_MODES = {"off": 0, "check": 1, "auto": 2}


class CandidateRecord(C.Structure):
    """ft_b200_candidate (ft_candidate, fainttrail.h:55-68)."""
    _fields_ = [("id", C.c_int), ("ok", C.c_int)] + [(n, C.c_double) for n in (
        "x", "y", "vx_pxh", "vy_pxh", "pos_err_px", "vel_err_pxh", "snr", "snr_coarse", "snr_half1", "snr_half2",
        "max_frame_fraction", "false_alarms_per_run", "flux", "mag_inst", "ra_deg", "dec_deg", "rate_arcsec_min",
        "pa_deg")] + [("flags", C.c_char * 64)]


class DriftCheck(C.Structure):
    """ft_b200_drift_check (DriftCheck, registration.hpp:22-30)."""
    _fields_ = [("measured", C.c_int), ("registered", C.c_int), ("stars", C.c_int), ("matched", C.c_int)] + [
        (n, C.c_double) for n in ("dx", "dy", "mid_dx", "mid_dy", "rate_pxh")] + [("message", C.c_char * 1024)]

    def as_dict(self):
        d = {k: getattr(self, k) for k in ("measured", "registered", "dx", "dy", "mid_dx", "mid_dy", "rate_pxh",
                                           "stars", "matched")}
        d["message"] = self.message.decode()
        return d


def _set_fields(struct, kw, what):
    """Set the named fields of a parameter struct; an unknown name is an error
    (ctypes would otherwise keep it as a plain attribute and ignore it)."""
    names = {f[0] for f in struct._fields_}
    unknown = sorted(set(kw) - names)
    if unknown:
        raise TypeError(f"unknown {what} parameter(s) {unknown}; known: {sorted(names)}")
    for k, v in kw.items():
        setattr(struct, k, v)


class Injection(C.Structure):
    """ft_b200_injection (Injection, validate.hpp:18-23)."""
    _fields_ = [(n, C.c_double) for n in ("x_ref", "y_ref", "vx_pxh", "vy_pxh", "flux")]


class Peak(C.Structure):
    _fields_ = [("x", C.c_int), ("y", C.c_int), ("snr", C.c_float), ("vidx", C.c_int)]


class Cancelled(RuntimeError):
    """A progress callback asked to stop (types.hpp:70-76)."""


def lib():
    """The loaded C ABI library (raises if it was not built)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(f"{LIB_PATH} is missing: build it with python -m fainttrail_b200.build")
            L = C.CDLL(LIB_PATH)
            _declare(L)
            _lib = L
    return _lib


def _declare(L):
    L.ft_b200_version.restype = C.c_char_p
    L.ft_b200_open.argtypes = [C.c_int, C.c_double, C.POINTER(C.c_void_p)]
    L.ft_b200_close.argtypes = [C.c_void_p]
    L.ft_b200_last_error.argtypes = [C.c_void_p]
    L.ft_b200_last_error.restype = C.c_char_p
    L.ft_b200_device_info.argtypes = [C.c_void_p, C.c_char_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double)]
    L.ft_b200_stack.argtypes = [C.c_void_p, _f32p, C.c_int, C.c_int, C.c_int, _i32p, _i32p, C.c_int, C.c_int,
                                _f32p, _i32p, PROGRESS_FN, C.c_void_p]
    L.ft_b200_stack_linear.argtypes = [C.c_void_p, _f32p, C.c_int, C.c_int, C.c_int, _f64p, _f64p, C.c_int, C.c_int,
                                       _f32p, _i32p, PROGRESS_FN, C.c_void_p]
    L.ft_b200_stack_dev.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, _i32p, _i32p, C.c_int,
                                    C.c_int, C.c_void_p, C.c_void_p]
    L.ft_b200_timings.argtypes = [C.c_void_p, C.c_char_p, C.c_int, C.c_void_p, C.c_int]
    L.ft_b200_stage_params_default.argtypes = [C.POINTER(StageParams)]
    L.ft_b200_search_params_default.argtypes = [C.POINTER(SearchParams)]
    L.ft_b200_search.argtypes = [C.c_void_p, _f32p, C.c_int, C.c_int, C.c_int, _f64p, _f64p, C.POINTER(SearchParams),
                                 PROGRESS_FN, C.c_void_p, C.POINTER(C.c_void_p)]
    L.ft_b200_search_tiled.argtypes = [C.c_void_p, _f32p, C.c_int, C.c_int, C.c_int, _f64p, _f64p,
                                       C.POINTER(SearchParams), C.c_int, PROGRESS_FN, C.c_void_p,
                                       C.POINTER(C.c_void_p)]
    L.ft_b200_search_dev.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, _f64p, _f64p,
                                     C.POINTER(SearchParams), C.POINTER(C.c_void_p)]
    L.ft_b200_stats.argtypes = [C.c_void_p, C.POINTER(C.c_longlong), C.POINTER(C.c_double)]
    L.ft_b200_search_batch.argtypes = [C.c_void_p, _f32p, C.c_int, C.c_int, C.c_int, _f64p, _f64p,
                                       C.POINTER(SearchParams), C.c_int, C.c_void_p, C.c_void_p, PROGRESS_FN,
                                       C.c_void_p, C.POINTER(C.c_void_p), C.c_void_p]
    L.ft_b200_search_batch_dev.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, _f64p, _f64p,
                                           C.POINTER(SearchParams), C.c_int, C.c_void_p, C.c_void_p,
                                           C.POINTER(C.c_void_p), C.c_void_p]
    L.ft_b200_result_free.argtypes = [C.c_void_p]
    L.ft_b200_plan_stats.argtypes = [C.c_int, C.c_int, C.c_int, _i32p, _i32p, C.c_int, C.c_int,
                                     np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")]
    L.ft_b200_emulate_stack.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, _i32p, _i32p, C.c_int, C.c_int, C.c_int,
                                        _f32p, _i32p]
    L.ft_b200_check_registration.argtypes = [C.c_void_p, _f32p, C.c_int, C.c_int, C.c_int, _f64p,
                                             C.POINTER(DriftCheck)]
    L.ft_b200_check_registration_dev.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, _f64p,
                                                 C.POINTER(DriftCheck)]
    L.ft_b200_result_registration.argtypes = [C.c_void_p, C.POINTER(DriftCheck)]
    L.ft_b200_result_candidates_csv.argtypes = [C.c_void_p, C.c_char_p, C.c_longlong]
    L.ft_b200_result_candidates_csv.restype = C.c_longlong
    L.ft_b200_write_candidates_csv.argtypes = [C.c_void_p, C.c_char_p]
    L.ft_b200_result_candidate.argtypes = [C.c_void_p, C.c_int, C.POINTER(CandidateRecord)]
    L.ft_b200_result_track_point.argtypes = [C.c_void_p, C.c_int, C.c_int] + [C.POINTER(C.c_double)] * 5
    L.ft_b200_result_candidates.argtypes = [C.c_void_p, C.c_void_p, C.c_char_p, C.c_int]
    L.ft_b200_result_threshold.argtypes = [C.c_void_p, C.c_char_p, C.c_int] + [C.POINTER(C.c_double)] * 4
    L.ft_b200_result_threshold.restype = C.c_double
    L.ft_b200_result_info.argtypes = [C.c_void_p] + [C.POINTER(C.c_double)] * 3 + [C.POINTER(C.c_int)]
    L.ft_b200_result_peaks.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int]
    L.ft_b200_result_null_peaks.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
    L.ft_b200_result_maps.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    L.ft_b200_result_velocity.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.ft_b200_stage.argtypes = [C.c_void_p, _f32p, C.c_int, C.c_int, C.c_int, _f64p, C.POINTER(StageParams),
                                C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.ft_b200_stage_dev.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, _f64p,
                                    C.POINTER(StageParams)] + [C.c_void_p] * 5


def _declare_server(L):
    L.ft_b200_server_open.argtypes = [C.c_int, C.c_double, C.c_int, C.c_int, C.POINTER(C.c_void_p)]
    L.ft_b200_server_close.argtypes = [C.c_void_p]
    L.ft_b200_server_submit.argtypes = [C.c_void_p, _f32p, C.c_int, C.c_int, C.c_int, _f64p, _f64p,
                                        C.POINTER(SearchParams), C.POINTER(C.c_longlong)]
    L.ft_b200_server_poll.argtypes = [C.c_void_p, C.c_longlong, C.c_int, C.POINTER(C.c_void_p)]
    L.ft_b200_server_error.argtypes = [C.c_void_p]
    L.ft_b200_server_error.restype = C.c_char_p
    L.ft_b200_server_pause.argtypes = [C.c_void_p, C.c_int]
    L.ft_b200_server_stats.argtypes = [C.c_void_p, C.POINTER(C.c_longlong), C.POINTER(C.c_double),
                                       C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_longlong),
                                       C.POINTER(C.c_double), C.POINTER(C.c_longlong)]


FT_B200_PENDING = 3


class Server:
    """The serving loop (ft_b200_server_*): submit searches at any time, poll
    results; requests admitted together share their stacking launches."""

    def __init__(self, device=-1, hbm_budget_bytes=0.0, max_batch=16, workers=2):
        self.L = lib()
        _declare_server(self.L)
        h = C.c_void_p()
        if self.L.ft_b200_server_open(device, hbm_budget_bytes, max_batch, workers, C.byref(h)) != FT_B200_OK:
            raise RuntimeError("ft_b200_server_open: " + self.L.ft_b200_last_error(None).decode())
        self.h = h
        self._dev = None

    def submit(self, frames, mjd, exptime, **kw):
        frames = np.ascontiguousarray(frames, dtype=np.float32)
        n, h, w = frames.shape
        p = Device._search_params(self.L, kw)
        rid = C.c_longlong()
        rc = self.L.ft_b200_server_submit(self.h, frames, w, h, n, np.ascontiguousarray(mjd, dtype=np.float64),
                                          np.ascontiguousarray(exptime, dtype=np.float64), C.byref(p), C.byref(rid))
        if rc != FT_B200_OK:
            raise RuntimeError("submit: " + self.L.ft_b200_server_error(self.h).decode())
        return rid.value, (w, h)

    def poll(self, ticket, wait_ms=-1, maps=True):
        rid, (w, h) = ticket
        r = C.c_void_p()
        rc = self.L.ft_b200_server_poll(self.h, rid, wait_ms, C.byref(r))
        if rc == FT_B200_PENDING:
            return None
        if rc != FT_B200_OK:
            raise RuntimeError("poll: " + self.L.ft_b200_server_error(self.h).decode())
        return _read_result(self.L, r, w, h, maps)

    def pause(self, paused=True):
        self.L.ft_b200_server_pause(self.h, 1 if paused else 0)

    def stats(self):
        c, r, nl = C.c_longlong(), C.c_longlong(), C.c_longlong()
        p50, p99, sps, mb = C.c_double(), C.c_double(), C.c_double(), C.c_double()
        self.L.ft_b200_server_stats(self.h, C.byref(c), C.byref(p50), C.byref(p99), C.byref(sps), C.byref(r),
                                    C.byref(mb), C.byref(nl))
        return dict(completed=c.value, p50_s=p50.value, p99_s=p99.value, searches_per_s=sps.value, rounds=r.value,
                    mean_batch=mb.value, launches=nl.value)

    def close(self):
        if getattr(self, "h", None):
            self.L.ft_b200_server_close(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class CompletenessRow(C.Structure):
    _fields_ = [("target_snr", C.c_double), ("injected", C.c_int), ("recovered", C.c_int), ("detected", C.c_int),
                ("mean_snr", C.c_double), ("mean_dpos", C.c_double), ("mean_dv", C.c_double)]


def completeness(device, frames, mjd, exptime, snr_levels=(4.0, 5.0, 6.0, 7.0, 8.0, 10.0, 12.0, 15.0), per_level=10,
                 min_separation=40.0, seed=99, **kw):
    """ft_b200_completeness (completeness(), validate.cpp:62-165) on `device` (a
    Device): returns dict(rows=[dict per level], threshold, method, baseline_ok,
    snr50)."""
    L = device.L
    L.ft_b200_completeness.argtypes = [C.c_void_p, _f32p, C.c_int, C.c_int, C.c_int, _f64p, _f64p,
                                       C.POINTER(SearchParams), _f64p, C.c_int, C.c_int, C.c_double, C.c_ulonglong,
                                       C.POINTER(CompletenessRow), C.POINTER(C.c_double), C.c_char_p, C.c_int,
                                       C.POINTER(C.c_int), C.POINTER(C.c_double)]
    frames = np.ascontiguousarray(frames, dtype=np.float32)
    n, h, w = frames.shape
    p = Device._search_params(L, kw)
    lv = np.ascontiguousarray(snr_levels, dtype=np.float64)
    rows = (CompletenessRow * max(1, lv.size))()
    thr, snr50 = C.c_double(), C.c_double()
    ok = C.c_int()
    meth = C.create_string_buffer(32)
    rc = L.ft_b200_completeness(device.h, frames, w, h, n, np.ascontiguousarray(mjd, dtype=np.float64),
                                np.ascontiguousarray(exptime, dtype=np.float64), C.byref(p), lv, lv.size, per_level,
                                min_separation, seed, rows, C.byref(thr), meth, 32, C.byref(ok), C.byref(snr50))
    device.check(rc, "completeness")
    out = [dict(target_snr=r.target_snr, injected=r.injected, recovered=r.recovered, detected=r.detected,
                mean_snr=r.mean_snr, mean_dpos=r.mean_dpos, mean_dv=r.mean_dv) for r in rows[:lv.size]]
    return dict(rows=out, threshold=thr.value, method=meth.value.decode(), baseline_ok=ok.value, snr50=snr50.value)


def plan_stats(w, h, n, dx, dy, shape=0):
    """ft_b200_plan_stats: the planner's motion groups for a pass (host only):
    dict(groups, row_groups, slots, pads, row_slots, max_group_bytes)."""
    L = lib()
    dx = np.ascontiguousarray(dx, dtype=np.int32)
    dy = np.ascontiguousarray(dy, dtype=np.int32)
    out = np.zeros(6, np.int64)
    if L.ft_b200_plan_stats(w, h, n, dx, dy, dx.size // n, shape, out) != FT_B200_OK:
        raise RuntimeError("plan_stats: " + L.ft_b200_last_error(None).decode())
    return dict(zip(("groups", "row_groups", "slots", "pads", "row_slots", "max_group_bytes"), map(int, out)))


def emulate_stack(frames, dx, dy, min_count, shape=0):
    """ft_b200_emulate_stack: one pass computed on the CPU as the device kernel
    computes it over its plan (for checks without a GPU). frames (n, h, w);
    dx/dy (m, n) motion-major shifts. Returns (max_snr, best_v)."""
    L = lib()
    frames = np.ascontiguousarray(frames, dtype=np.float32)
    n, h, w = frames.shape
    dx = np.ascontiguousarray(dx, dtype=np.int32)
    dy = np.ascontiguousarray(dy, dtype=np.int32)
    m = dx.size // n
    ms = np.empty((h, w), np.float32)
    bv = np.empty((h, w), np.int32)
    if L.ft_b200_emulate_stack(frames, w, h, n, dx, dy, m, min_count, shape, ms, bv) != FT_B200_OK:
        raise RuntimeError("emulate_stack: " + L.ft_b200_last_error(None).decode())
    return ms, bv


def set_tile_shape(shape):
    """ft_b200_set_tile_shape: 0 automatic, 1 = 32 x 16, 2 = 64 x 8 paired
    columns, 3 = 32 x 8, 4 = 32 x 4, 5 / 6 = 32 x 16 with one shared maximum per
    tile (16 / 14 warps), 7 = 32 x 12 (16 warps), 8 = 32 x 20 with the shared
    maximum (16 warps); process-wide."""
    L = lib()
    L.ft_b200_set_tile_shape.argtypes = [C.c_int]
    if L.ft_b200_set_tile_shape(int(shape)) != FT_B200_OK:
        raise ValueError("ft_b200_set_tile_shape: " + L.ft_b200_last_error(None).decode())


def tile_shape():
    return lib().ft_b200_tile_shape()


def tuned_shapes():
    """The autotuner's cache: {(frames, motions, width, height): shape}."""
    L = lib()
    cnt = L.ft_b200_tuned_shapes(None, None, 0)
    keys = (C.c_int * max(1, 4 * cnt))()
    shapes = (C.c_int * max(1, cnt))()
    L.ft_b200_tuned_shapes(keys, shapes, cnt)
    return {tuple(keys[4 * k:4 * k + 4]): shapes[k] for k in range(cnt)}


def clear_tuned_shapes():
    lib().ft_b200_clear_tuned_shapes()


def null_threshold(pooled, runs, psf_fwhm_px, width, height, motions, **kw):
    """ft_b200_null_threshold: the null-tail threshold from pooled null-peak S/N
    values (host only; no GPU), with the search's PSF width (a result's "fwhm")
    and search parameters **kw. Returns a dict like a search result's threshold
    fields."""
    L = lib()
    L.ft_b200_null_threshold.argtypes = [C.c_void_p, C.c_longlong, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int,
                                         C.POINTER(SearchParams), C.POINTER(C.c_double), C.c_char_p, C.c_int,
                                         C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double),
                                         C.POINTER(C.c_double)]
    p = Device._search_params(L, kw)
    v = np.ascontiguousarray(pooled, dtype=np.float64)
    thr, a, b, k, s2 = (C.c_double() for _ in range(5))
    meth = C.create_string_buffer(32)
    rc = L.ft_b200_null_threshold(v.ctypes.data_as(C.c_void_p), v.size, runs, psf_fwhm_px, width, height, motions,
                                  C.byref(p), C.byref(thr), meth, 32, C.byref(a), C.byref(b), C.byref(k), C.byref(s2))
    if rc != FT_B200_OK:
        raise RuntimeError("ft_b200_null_threshold: " + L.ft_b200_last_error(None).decode())
    return dict(threshold=thr.value, method=meth.value.decode(), null_a=a.value, null_b=b.value, null_k=k.value,
                null_inv_s2=s2.value)


def exported_symbols():
    """Names of the entry points include/ft_b200.h declares."""
    import re
    with open(os.path.join(os.path.dirname(HERE), "include", "ft_b200.h")) as f:
        text = f.read()
    return sorted(set(re.findall(r"\b(ft_b200_[a-z0-9_]+)\s*\(", text)))


class Device:
    """An open B200 context (ft_b200_open). One per host thread."""

    def __init__(self, device=-1, hbm_budget_bytes=0.0):
        self.L = lib()
        h = C.c_void_p()
        if self.L.ft_b200_open(device, hbm_budget_bytes, C.byref(h)) != FT_B200_OK:
            raise RuntimeError("ft_b200_open: " + self.L.ft_b200_last_error(None).decode())
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.ft_b200_close(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def error(self):
        return self.L.ft_b200_last_error(self.h).decode()

    def check(self, rc, what):
        if rc == FT_B200_CANCELLED:
            raise Cancelled("cancelled")
        if rc != FT_B200_OK:
            raise RuntimeError(f"{what}: {self.error()}")

    def timings(self):
        """[(stage, seconds)] of the last call (CUDA events on the context stream)."""
        names = C.create_string_buffer(4096)
        vals = np.zeros(64)
        k = self.L.ft_b200_timings(self.h, names, 4096, vals.ctypes.data_as(C.c_void_p), 64)
        return list(zip(names.value.decode().split(";"), vals[:k].tolist())) if k else []

    def stack_dev(self, d_frames, width, height, pitch, nframes, dx, dy, min_count, d_max_snr, d_best_v):
        """ft_b200_stack_dev on device pointers (ints), host shift tables."""
        dx = np.ascontiguousarray(dx, dtype=np.int32)
        dy = np.ascontiguousarray(dy, dtype=np.int32)
        rc = self.L.ft_b200_stack_dev(self.h, C.c_void_p(d_frames), width, height, pitch, nframes, dx, dy,
                                      dx.shape[0], min_count, C.c_void_p(d_max_snr), C.c_void_p(d_best_v))
        self.check(rc, "stack_dev")

    def stage(self, sub, t_h, fwhm_px, **kw):
        """build_stage on host frames (ft_b200_stage). Returns a dict with
        filtered, static_sky, mask, sigma, cr (the reference's Prepared fields)."""
        sub = np.ascontiguousarray(sub, dtype=np.float32)
        n, h, w = sub.shape
        p = StageParams()
        self.L.ft_b200_stage_params_default(C.byref(p))
        p.fwhm_px = fwhm_px
        _set_fields(p, kw, "stage")
        filt = np.empty_like(sub)
        sky = np.empty((h, w), np.float32)
        mask = np.empty((h, w), np.float32)
        sigma = np.empty(n, np.float64)
        cr = np.empty(n, np.int32)
        ptr = lambda a: a.ctypes.data_as(C.c_void_p)
        rc = self.L.ft_b200_stage(self.h, sub, w, h, n, np.ascontiguousarray(t_h, dtype=np.float64), C.byref(p),
                                  ptr(filt), ptr(sky), ptr(mask), ptr(sigma), ptr(cr))
        self.check(rc, "stage")
        return dict(filtered=filt, static_sky=sky, mask=mask, sigma=sigma, cr=cr)

    def stage_dev(self, d_sub, width, height, pitch, nframes, t_h, fwhm_px, d_filtered=None, d_static_sky=None,
                  d_mask=None, **kw):
        """build_stage on device frames (ft_b200_stage_dev): d_sub and the
        outputs are device pointers with rows `pitch` floats apart (outputs may be
        None). Returns dict(sigma, cr)."""
        p = StageParams()
        self.L.ft_b200_stage_params_default(C.byref(p))
        p.fwhm_px = fwhm_px
        _set_fields(p, kw, "stage")
        sigma = np.empty(nframes, np.float64)
        cr = np.empty(nframes, np.int32)
        rc = self.L.ft_b200_stage_dev(self.h, C.c_void_p(d_sub), width, height, pitch, nframes,
                                      np.ascontiguousarray(t_h, dtype=np.float64), C.byref(p),
                                      C.c_void_p(d_filtered), C.c_void_p(d_static_sky), C.c_void_p(d_mask),
                                      sigma.ctypes.data_as(C.c_void_p), cr.ctypes.data_as(C.c_void_p))
        self.check(rc, "stage_dev")
        return dict(sigma=sigma, cr=cr)

    def launches(self):
        """Kernels launched by the last call (ft_b200_stats)."""
        k = C.c_longlong()
        self.L.ft_b200_stats(self.h, C.byref(k), None)
        return k.value

    @staticmethod
    def _search_params(L, kw):
        p = SearchParams()
        L.ft_b200_search_params_default(C.byref(p))
        kw = dict(kw)
        if "calibrated_tail" in kw:
            kw["calibrated_tail"] = (C.c_double * 4)(*kw["calibrated_tail"])
        if isinstance(kw.get("align"), str):
            if kw["align"] not in ALIGN_MODES:
                raise ValueError(f"align must be one of {sorted(ALIGN_MODES)} (this backend does not resample "
                                 f"frames, so 'always' has no counterpart), not {kw['align']!r}")
            kw["align"] = ALIGN_MODES[kw["align"]]
        # per-frame registration offsets: arrays kept alive with the parameters
        reg = [kw.pop(k, None) for k in ("reg_dx", "reg_dy")]
        if (reg[0] is None) != (reg[1] is None):
            raise ValueError("registration offsets need both reg_dx and reg_dy")
        _set_fields(p, kw, "search")
        if reg[0] is not None:
            p._reg = [np.ascontiguousarray(a, dtype=np.float64) for a in reg]
            p.reg_dx = p._reg[0].ctypes.data_as(C.c_void_p)
            p.reg_dy = p._reg[1].ctypes.data_as(C.c_void_p)
        return p

    def check_registration(self, frames, t_h):
        """The registration check (ft_b200_check_registration) of frames
        (n, h, w) observed at t_h hours; returns the DriftCheck as a dict."""
        frames = np.ascontiguousarray(frames, dtype=np.float32)
        n, h, w = frames.shape
        out = DriftCheck()
        rc = self.L.ft_b200_check_registration(self.h, frames, w, h, n, np.ascontiguousarray(t_h, dtype=np.float64),
                                               C.byref(out))
        self.check(rc, "check_registration")
        return out.as_dict()

    def check_registration_dev(self, d_frames, width, height, pitch, nframes, t_h):
        """ft_b200_check_registration_dev on a device pointer."""
        out = DriftCheck()
        rc = self.L.ft_b200_check_registration_dev(self.h, C.c_void_p(d_frames), width, height, pitch, nframes,
                                                   np.ascontiguousarray(t_h, dtype=np.float64), C.byref(out))
        self.check(rc, "check_registration_dev")
        return out.as_dict()

    def search_dev(self, d_frames, width, height, pitch, nframes, mjd, exptime, maps=True, **kw):
        """ft_b200_search_dev on a device pointer; returns the result dict."""
        p = self._search_params(self.L, kw)
        r = C.c_void_p()
        rc = self.L.ft_b200_search_dev(self.h, C.c_void_p(d_frames), width, height, pitch, nframes,
                                       np.ascontiguousarray(mjd, dtype=np.float64),
                                       np.ascontiguousarray(exptime, dtype=np.float64), C.byref(p), C.byref(r))
        self.check(rc, "search_dev")
        return self._result(r, width, height, maps)

    def search(self, frames, mjd, exptime, progress=None, maps=True, csv_path=None, **kw):
        """A whole search (ft_b200_search) from raw frames; returns a dict
        (threshold and tail fit, peaks, maps, null peaks, candidates with their
        track points, the candidate file's text, the registration check). kw are
        ft_b200_search_params fields (align: "off", "check" or "auto"). With
        csv_path, the candidate file is also written there
        (ft_b200_write_candidates_csv)."""
        frames = np.ascontiguousarray(frames, dtype=np.float32)
        n, h, w = frames.shape
        p = self._search_params(self.L, kw)
        r = C.c_void_p()
        rc = self.L.ft_b200_search(self.h, frames, w, h, n, np.ascontiguousarray(mjd, dtype=np.float64),
                                   np.ascontiguousarray(exptime, dtype=np.float64), C.byref(p), _progress(progress),
                                   None, C.byref(r))
        self.check(rc, "search")
        return self._result(r, w, h, maps, csv_path)

    def search_tiled(self, frames, mjd, exptime, band_rows=0, progress=None, maps=True, **kw):
        """The tiled search (ft_b200_search_tiled): the frames stay in host
        memory and go to the device in bands of band_rows rows (0: 1024) with
        their halos; the result equals search()'s."""
        frames = np.ascontiguousarray(frames, dtype=np.float32)
        n, h, w = frames.shape
        p = self._search_params(self.L, kw)
        r = C.c_void_p()
        rc = self.L.ft_b200_search_tiled(self.h, frames, w, h, n, np.ascontiguousarray(mjd, dtype=np.float64),
                                         np.ascontiguousarray(exptime, dtype=np.float64), C.byref(p), int(band_rows),
                                         _progress(progress), None, C.byref(r))
        self.check(rc, "search_tiled")
        return self._result(r, w, h, maps)

    def search_batch(self, frames, mjd, exptime, copies, progress=None, maps=True, **kw):
        """ft_b200_search_batch: the search plus injection copies. `copies` is a
        list of lists of (x_ref, y_ref, vx_pxh, vy_pxh, flux). Returns (base
        result dict, [copy result dicts])."""
        frames = np.ascontiguousarray(frames, dtype=np.float32)
        n, h, w = frames.shape
        p = self._search_params(self.L, kw)
        counts = (C.c_int * max(1, len(copies)))(*[len(c) for c in copies])
        flat = [o for c in copies for o in c]
        objs = (Injection * max(1, len(flat)))(*[Injection(*o) for o in flat])
        base = C.c_void_p()
        outs = (C.c_void_p * max(1, len(copies)))()
        rc = self.L.ft_b200_search_batch(self.h, frames, w, h, n, np.ascontiguousarray(mjd, dtype=np.float64),
                                         np.ascontiguousarray(exptime, dtype=np.float64), C.byref(p), len(copies),
                                         counts, objs, _progress(progress), None, C.byref(base), outs)
        self.check(rc, "search_batch")
        res = self._result(base, w, h, maps)
        return res, [self._result(C.c_void_p(outs[k]), w, h, maps) for k in range(len(copies))]

    def search_batch_dev(self, d_frames, width, height, pitch, nframes, mjd, exptime, copies, maps=True, **kw):
        """ft_b200_search_batch_dev: search_batch over frames in device memory."""
        p = self._search_params(self.L, kw)
        counts = (C.c_int * max(1, len(copies)))(*[len(c) for c in copies])
        flat = [o for c in copies for o in c]
        objs = (Injection * max(1, len(flat)))(*[Injection(*o) for o in flat])
        base = C.c_void_p()
        outs = (C.c_void_p * max(1, len(copies)))()
        rc = self.L.ft_b200_search_batch_dev(self.h, C.c_void_p(d_frames), width, height, pitch, nframes,
                                             np.ascontiguousarray(mjd, dtype=np.float64),
                                             np.ascontiguousarray(exptime, dtype=np.float64), C.byref(p),
                                             len(copies), counts, objs, C.byref(base), outs)
        self.check(rc, "search_batch_dev")
        res = self._result(base, width, height, maps)
        return res, [self._result(C.c_void_p(outs[k]), width, height, maps) for k in range(len(copies))]

    def _result(self, r, w, h, maps, csv_path=None):
        return _read_result(self.L, r, w, h, maps, csv_path)

    def info(self):
        name = C.create_string_buffer(256)
        sms, mem = C.c_int(), C.c_double()
        self.check(self.L.ft_b200_device_info(self.h, name, 256, C.byref(sms), C.byref(mem)), "device_info")
        return name.value.decode(), sms.value, mem.value


def _read_result(L, r, w, h, maps, csv_path=None):
    """The getters of an ft_b200_result (freed here) as a dict; with csv_path,
    the candidate file is written there first."""
    try:
        if csv_path is not None and L.ft_b200_write_candidates_csv(r, os.fsencode(csv_path)) != FT_B200_OK:
            raise RuntimeError(L.ft_b200_last_error(None).decode())
        meth = C.create_string_buffer(32)
        a, b, k, s2 = C.c_double(), C.c_double(), C.c_double(), C.c_double()
        thr = L.ft_b200_result_threshold(r, meth, 32, C.byref(a), C.byref(b), C.byref(k), C.byref(s2))
        fw, dv, tref, nv = C.c_double(), C.c_double(), C.c_double(), C.c_int()
        L.ft_b200_result_info(r, C.byref(fw), C.byref(dv), C.byref(tref), C.byref(nv))

        def peaks(which):
            cnt = L.ft_b200_result_peaks(r, which, None, 0)
            arr = (Peak * max(cnt, 1))()
            L.ft_b200_result_peaks(r, which, arr, cnt)
            return [(q.x, q.y, q.snr, q.vidx) for q in arr[:cnt]]
        cnt = L.ft_b200_result_null_peaks(r, None, 0)
        nulls = np.empty(cnt)
        L.ft_b200_result_null_peaks(r, nulls.ctypes.data_as(C.c_void_p), cnt)
        ms = bv = None
        if maps:
            ms = np.empty((h, w), np.float32)
            bv = np.empty((h, w), np.int32)
            if L.ft_b200_result_maps(r, ms.ctypes.data_as(C.c_void_p), bv.ctypes.data_as(C.c_void_p)) != FT_B200_OK:
                ms = bv = None  # a null-run shard other than 0 has no maps
        grid = np.empty((nv.value, 2))
        vx, vy = C.c_double(), C.c_double()
        for j in range(nv.value):
            L.ft_b200_result_velocity(r, j, C.byref(vx), C.byref(vy))
            grid[j] = (vx.value, vy.value)
        nc = L.ft_b200_result_candidates(r, None, None, 0)
        rows = np.empty((max(nc, 1), 17))
        fl = C.create_string_buffer(64 * max(nc, 1))
        L.ft_b200_result_candidates(r, rows.ctypes.data_as(C.c_void_p), fl, nc)
        cands = [(rows[q].copy(), fl.raw[64 * q:64 * q + 64].split(b"\0", 1)[0].decode()) for q in range(nc)]
        reg = DriftCheck()
        L.ft_b200_result_registration(r, C.byref(reg))
        pt = [C.c_double() for _ in range(5)]
        tracks = []
        for q in range(nc):  # every frame of every candidate (ft_get_track_point)
            f, rows_q = 0, []
            while L.ft_b200_result_track_point(r, q, f, *[C.byref(v) for v in pt]) == FT_B200_OK:
                rows_q.append([v.value for v in pt])
                f += 1
            tracks.append(rows_q)
        track_points = np.array(tracks, np.float64).reshape(nc, -1, 5) if nc else np.zeros((0, 0, 5))
        size = L.ft_b200_result_candidates_csv(r, None, 0)
        text = C.create_string_buffer(size + 1)
        L.ft_b200_result_candidates_csv(r, text, size + 1)
        return dict(threshold=thr, method=meth.value.decode(), null_a=a.value, null_b=b.value, null_k=k.value,
                    null_inv_s2=s2.value, fwhm=fw.value, dv=dv.value, t_ref=tref.value, n_velocities=nv.value,
                    peaks=peaks(0), selected=peaks(1), null_peaks=nulls, max_snr=ms, best_v=bv, grid=grid,
                    candidates=cands, registration=reg.as_dict(), candidates_csv=text.value.decode(),
                    track_points=track_points)
    finally:
        L.ft_b200_result_free(r)


def _progress(fn):
    if fn is None:
        return PROGRESS_FN()

    def cb(f, stage, _user):
        return 1 if fn(f, stage.decode() if stage else "") else 0
    return PROGRESS_FN(cb)


# ----------------------------------------------------------------------------- plugin mirror
class StackPass:
    """One stacking pass (backend.hpp:71-78): frames (n, h, w) float32, either
    times t_h + velocities (m, 2) or an explicit shift table (dx, dy: (m, n))."""

    def __init__(self, frames, t_h=None, velocities=None, shifts=None, min_count=3, threads=0):
        self.frames = frames
        self.t_h = t_h
        self.velocities = velocities
        self.shifts = shifts
        self.min_count = min_count
        self.threads = threads


class StackResult:
    """max_snr (h, w) float32, best_v (h, w) int32 (backend.hpp:99-105)."""

    def __init__(self, max_snr, best_v, timings=None):
        self.max_snr = max_snr
        self.best_v = best_v
        self.timings = timings or []


def validate_pass(p):
    """The checks of validate_pass (backend.cpp:89-108); raises RuntimeError."""
    if p.frames is None:
        raise RuntimeError("stack pass: missing frames")
    f = np.asarray(p.frames)
    if f.ndim != 3 or f.shape[0] == 0:
        raise RuntimeError("stack pass: no frames")
    n = f.shape[0]
    if p.shifts is not None:
        dx, dy = (np.asarray(a) for a in p.shifts)
        if dx.ndim != 2 or dx.shape[1] != n:
            raise RuntimeError("stack pass: shift table and frame counts differ")
        if dx.shape[0] < 1 or dy.shape != dx.shape:
            raise RuntimeError("stack pass: malformed shift table")
        if p.velocities is not None and len(p.velocities) != dx.shape[0]:
            raise RuntimeError("stack pass: shift table and velocity counts differ")
    else:
        if p.t_h is None or p.velocities is None:
            raise RuntimeError("stack pass: missing times or velocities")
        if len(p.t_h) != n:
            raise RuntimeError("stack pass: frame and time counts differ")
    if p.min_count < 1:
        raise RuntimeError("stack pass: min_count must be at least 1")


class SearchBackend:
    """The "b200" stacking backend (SearchBackend, backend.hpp:107-117)."""

    def __init__(self, device=None):
        self.dev = device if device is not None else Device()

    def name(self):
        return "b200"

    def description(self):
        name, sms, mem = self.dev.info()
        return f"B200 backend: {name}, {mem / 1073741824.0:.1f} GB, {sms} SMs, sm_100a kernels"

    def run(self, p, progress=None):
        validate_pass(p)
        frames = np.ascontiguousarray(p.frames, dtype=np.float32)
        n, h, w = frames.shape
        ms = np.empty((h, w), np.float32)
        bv = np.empty((h, w), np.int32)
        cb = _progress(progress)
        if p.shifts is not None:
            dx = np.ascontiguousarray(p.shifts[0], dtype=np.int32)
            dy = np.ascontiguousarray(p.shifts[1], dtype=np.int32)
            rc = self.dev.L.ft_b200_stack(self.dev.h, frames, w, h, n, dx, dy, dx.shape[0], p.min_count, ms, bv, cb,
                                          None)
        else:
            t = np.ascontiguousarray(p.t_h, dtype=np.float64)
            v = np.ascontiguousarray(p.velocities, dtype=np.float64).reshape(-1, 2)
            rc = self.dev.L.ft_b200_stack_linear(self.dev.h, frames, w, h, n, t, v, v.shape[0], p.min_count, ms, bv,
                                                 cb, None)
        self.dev.check(rc, "stack")
        return StackResult(ms, bv)


def make_backend(name="b200", device=None):
    """make_backend (backend.hpp:139) for this package's one backend."""
    if name != "b200":
        raise RuntimeError(f"unknown or unavailable search backend '{name}' (available: b200)")
    return SearchBackend(device)
