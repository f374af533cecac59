"""ctypes bindings for the test checkers under oracle/ (test infrastructure only).

* ``Oracle``: the C++ restatement of the reference's hot path (oracle/libft_oracle.so).
* ``Reference``: the reference library itself, built from its own sources by
  oracle/Makefile into oracle/_ref/ (present where that build ran).
"""
import ctypes as C
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "libft_oracle.so")
REF_DRIVER_SO = os.path.join(ROOT, "oracle", "_ref", "libftref_driver.so")

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class StageParams(C.Structure):
    _fields_ = [("fwhm_px", C.c_double), ("static_exclude", C.c_int), ("clip_sigma", C.c_double),
                ("cr_sigma", C.c_double), ("mask_scatter", C.c_double), ("weight_scatter", C.c_double)]


def stage_params(fwhm_px, static_exclude=-1, clip_sigma=8.0, cr_sigma=5.0, mask_scatter=2.5, weight_scatter=1.5):
    return StageParams(fwhm_px, static_exclude, clip_sigma, cr_sigma, mask_scatter, weight_scatter)


class Oracle:
    def __init__(self, path=ORACLE_SO):
        if not os.path.exists(path):
            raise RuntimeError(f"oracle library missing: {path} (run make -C oracle)")
        L = self.L = C.CDLL(path)
        L.fto_stack.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, _i32p, _i32p, C.c_int, C.c_int, _f32p, _i32p]
        L.fto_build_stage.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, _f64p, C.POINTER(StageParams),
                                      _f32p, _f32p, _f32p, _f64p, _i32p, C.c_void_p]
        L.fto_velocity_grid.argtypes = [C.c_double, C.c_double, C.c_double, C.c_double, C.c_void_p, C.c_int,
                                        C.POINTER(C.c_double)]
        L.fto_velocity_grid.restype = C.c_int
        L.fto_shift_table.argtypes = [_f64p, C.c_int, _f64p, C.c_int, _i32p, _i32p]
        L.fto_min_count.argtypes = [C.c_double, C.c_int]
        L.fto_null_orders.argtypes = [_f64p, C.c_int, C.c_int, C.c_ulonglong, _f64p]
        L.fto_find_peaks.argtypes = [_f32p, _i32p, C.c_int, C.c_int, C.c_float, C.c_int, C.c_int, C.c_int,
                                     _i32p, _i32p, _f32p, _i32p]
        L.fto_find_peaks.restype = C.c_int
        L.fto_is_artefact_peak.argtypes = [_f32p, _f32p, _f32p, _f64p, C.c_int, C.c_int, C.c_int, C.c_double,
                                           C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_void_p,
                                           C.c_void_p]
        L.fto_set_threshold.argtypes = [_f32p, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int,
                                        C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_double),
                                        C.POINTER(C.c_double)]
        L.fto_set_threshold.restype = C.c_double
        L.fto_median.argtypes = [_f32p, C.c_size_t]
        L.fto_median.restype = C.c_double
        L.fto_robust_sigma.argtypes = [_f32p, C.c_size_t]
        L.fto_robust_sigma.restype = C.c_double
        L.fto_background.argtypes = [_f32p, C.c_int, C.c_int]
        L.fto_background.restype = C.c_double
        L.fto_subtract_and_grow.argtypes = [_f32p, C.c_int, C.c_int, C.c_double, _f32p]

    def stack(self, frames, dx, dy, min_count):
        frames = _f32(frames)
        n, h, w = frames.shape
        dx, dy = _i32(dx), _i32(dy)
        m = dx.size // n
        ms = np.empty((h, w), np.float32)
        bv = np.empty((h, w), np.int32)
        self.L.fto_stack(frames, w, h, n, dx, dy, m, min_count, ms, bv)
        return ms, bv

    def build_stage(self, sub, t_h, fwhm_px, **kw):
        sub = _f32(sub)
        n, h, w = sub.shape
        sp = stage_params(fwhm_px, **kw)
        filt = np.empty_like(sub)
        sky = np.empty((h, w), np.float32)
        mask = np.empty((h, w), np.float32)
        sigma = np.empty(n, np.float64)
        cr = np.empty(n, np.int32)
        scatter = np.empty((h, w), np.float32)
        self.L.fto_build_stage(sub, w, h, n, _f64(t_h), C.byref(sp), filt, sky, mask, sigma, cr,
                               scatter.ctypes.data_as(C.c_void_p))
        return dict(filtered=filt, static_sky=sky, mask=mask, sigma=sigma, cr=cr, scatter=scatter)

    def velocity_grid(self, span_h, vmin, vmax, grid_tol):
        dv = C.c_double()
        cnt = self.L.fto_velocity_grid(span_h, vmin, vmax, grid_tol, None, 0, C.byref(dv))
        out = np.empty((max(cnt, 0), 2), np.float64)
        self.L.fto_velocity_grid(span_h, vmin, vmax, grid_tol, out.ctypes.data_as(C.c_void_p), cnt, C.byref(dv))
        return out, dv.value

    def shift_table(self, t_h, vel):
        t_h, vel = _f64(t_h), _f64(vel)
        n, m = t_h.size, vel.shape[0]
        dx = np.empty((m, n), np.int32)
        dy = np.empty((m, n), np.int32)
        self.L.fto_shift_table(t_h, n, vel, m, dx, dy)
        return dx, dy

    def min_count(self, min_coverage, n):
        return self.L.fto_min_count(min_coverage, n)

    def null_orders(self, t_h, runs, seed):
        t_h = _f64(t_h)
        out = np.empty((runs, t_h.size), np.float64)
        self.L.fto_null_orders(t_h, t_h.size, runs, seed, out)
        return out

    def find_peaks(self, max_snr, best_v, floor, radius, edge, max_peaks):
        max_snr, best_v = _f32(max_snr), _i32(best_v)
        h, w = max_snr.shape
        cap = max(1, w * h)
        px, py, pv = (np.empty(cap, np.int32) for _ in range(3))
        ps = np.empty(cap, np.float32)
        k = self.L.fto_find_peaks(max_snr, best_v, w, h, floor, radius, edge, max_peaks, px, py, ps, pv)
        return px[:k], py[:k], ps[:k], pv[:k]

    def is_artefact_peak(self, filtered, sub, static_sky, t_h, fwhm, x, y, vx, vy, max_frame_fraction=0.25):
        filtered, sub, sky = _f32(filtered), _f32(sub), _f32(static_sky)
        n, h, w = filtered.shape
        return self.L.fto_is_artefact_peak(filtered, sub, sky, _f64(t_h), n, w, h, fwhm, x, y, vx, vy,
                                           max_frame_fraction, None, None)

    def set_threshold(self, pooled, runs, target=0.02, floor=5.0, gauss=True):
        pooled = _f32(pooled)
        meth, a, k, s2 = C.c_int(), C.c_double(), C.c_double(), C.c_double()
        thr = self.L.fto_set_threshold(pooled, pooled.size, runs, target, floor, int(gauss), C.byref(meth),
                                       C.byref(a), C.byref(k), C.byref(s2))
        return thr, meth.value, a.value, k.value, s2.value

    def median(self, v):
        v = _f32(np.array(v, np.float32, copy=True))
        return self.L.fto_median(v, v.size)

    def robust_sigma(self, v):
        v = _f32(np.array(v, np.float32, copy=True))
        return self.L.fto_robust_sigma(v, v.size)

    def prepare_sub(self, raw):
        raw = _f32(raw)
        n, h, w = raw.shape
        sub = np.empty_like(raw)
        bgs = np.empty(n)
        for i in range(n):
            bgs[i] = self.L.fto_background(raw[i], w, h)
            out = np.empty((h, w), np.float32)
            self.L.fto_subtract_and_grow(_f32(raw[i]), w, h, bgs[i], out)
            sub[i] = out
        return sub, bgs


# ----------------------------------------------------------------------------- reference
class FtParams(C.Structure):
    """The reference's C API parameter struct (fainttrail.h:32-54)."""
    _fields_ = [(n, C.c_double) for n in (
        "vmin_pxh", "vmax_pxh", "grid_tol_px", "fwhm_px", "clip_sigma", "cr_sigma", "mask_scatter",
        "weight_scatter", "min_coverage", "threshold_snr", "min_snr_floor", "target_false_per_run",
        "max_frame_fraction", "half_tolerance")] + [
        ("static_exclude", C.c_int), ("null_runs", C.c_int), ("max_candidates", C.c_int), ("edge_px", C.c_int),
        ("threads", C.c_int), ("seed", C.c_ulonglong), ("backend", C.c_char * 16)]


class SimParams(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("width", "height", "nframes", "nstars", "nmovers", "hot_pixels")] + [
        (n, C.c_double) for n in (
            "exptime_s", "cadence_s", "fwhm_px", "sky_e_per_s", "read_noise_e", "gain_e_per_adu", "bias_adu",
            "rate_min_arcsec_min", "rate_max_arcsec_min", "pixscale_arcsec", "cosmic_rays_per_frame",
            "fwhm_jitter", "transparency_jitter", "star_mag_bright", "star_mag_faint")] + [
        ("seed", C.c_ulonglong)]


class Reference:
    def __init__(self, path=REF_DRIVER_SO):
        if not os.path.exists(path):
            raise RuntimeError(f"reference build missing: {path} (run make -C oracle ref)")
        L = self.L = C.CDLL(path, mode=C.RTLD_GLOBAL)
        L.ftref_last_error.restype = C.c_char_p
        L.ftref_simulate.argtypes = [C.POINTER(SimParams), _f32p, _f64p, _f64p]
        L.ftref_simulate_movers.argtypes = [C.POINTER(SimParams), _f64p, C.c_int, _f32p, _f64p, _f64p]
        L.ftref_prepare.argtypes = [C.c_int, C.c_int, C.c_int, _f32p, _f64p, _f64p, C.POINTER(FtParams)]
        L.ftref_prepare.restype = C.c_void_p
        L.ftref_prepare_reg.argtypes = [C.c_int, C.c_int, C.c_int, _f32p, _f64p, _f64p, C.c_void_p, C.c_void_p,
                                        C.POINTER(FtParams)]
        L.ftref_prepare_reg.restype = C.c_void_p
        L.ftref_load_frames.argtypes = [C.c_char_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                        C.POINTER(C.c_int)]
        L.ftref_prep_free.argtypes = [C.c_void_p]
        L.ftref_prep_info.argtypes = [C.c_void_p] + [C.POINTER(C.c_int)] * 3 + [C.POINTER(C.c_double)] * 3
        L.ftref_prep_vectors.argtypes = [C.c_void_p] + [C.c_void_p] * 5
        L.ftref_prep_images.argtypes = [C.c_void_p] + [C.c_void_p] * 4
        L.ftref_build_stage.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, _f64p, C.c_double, C.POINTER(FtParams),
                                        _f32p, _f32p, _f32p, _f64p, _i32p, C.c_void_p]
        L.ftref_stack.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.c_int, C.c_int, C.c_int, C.c_int, _f32p, _i32p]
        L.ftref_stack_cuda_timed.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, _f64p, _f64p, C.c_int, C.c_int,
                                             _f32p, _i32p, _f64p]
        L.ftref_check_backend.argtypes = [C.c_char_p, C.c_char_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.ftref_velocity_grid.argtypes = [C.c_double, C.POINTER(FtParams), C.c_void_p, C.c_int,
                                          C.POINTER(C.c_double)]
        L.ftref_null_orders.argtypes = [_f64p, C.c_int, C.c_int, C.c_ulonglong, _f64p]
        L.ftref_find_peaks.argtypes = [_f32p, _i32p, C.c_int, C.c_int, C.c_float, C.c_int, C.c_int, C.c_int,
                                       _i32p, _i32p, _f32p, _i32p]
        L.ftref_set_threshold.argtypes = [_f32p, C.c_int, C.c_int, C.POINTER(FtParams), C.c_char_p,
                                          C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.ftref_set_threshold.restype = C.c_double
        L.ftref_is_artefact_peak.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_int, C.c_double,
                                             C.c_double, C.POINTER(FtParams)]
        L.ftref_with_times.argtypes = [C.c_void_p, _f64p, C.POINTER(FtParams)]
        L.ftref_with_times.restype = C.c_void_p
        L.ftref_search.argtypes = [C.c_void_p, C.POINTER(FtParams)]
        L.ftref_search.restype = C.c_void_p
        L.ftref_check_registration.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, _f64p, _f64p, C.c_char_p, C.c_int]
        L.ftref_result_csv.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.ftref_iso_from_mjd.argtypes = [C.c_double, C.c_int, C.c_char_p, C.c_int]
        L.ftref_track_point.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, _f64p]
        L.ftref_result_free.argtypes = [C.c_void_p]
        L.ftref_result_scalars.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(C.c_double)] + \
            [C.POINTER(C.c_int)] * 3 + [C.POINTER(C.c_double)] * 3
        L.ftref_result_scalars.restype = C.c_double
        L.ftref_result_arrays.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.ftref_result_candidate.argtypes = [C.c_void_p, C.c_int, _f64p, C.c_char_p]
        L.ftref_inject.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, _f64p, _f64p, _f64p, C.c_int, C.c_double,
                                   C.c_double]
        if hasattr(L, "ftref_completeness"):
            L.ftref_completeness.argtypes = [C.c_int, C.c_int, C.c_int, _f32p, _f64p, _f64p, C.c_void_p, _f64p,
                                             C.c_int, C.c_int, C.c_double, C.c_ulonglong, C.c_void_p,
                                             C.POINTER(C.c_double), C.c_char_p, C.POINTER(C.c_int),
                                             C.POINTER(C.c_double)]

    def err(self):
        return self.L.ftref_last_error().decode()

    def params(self, **kw):
        p = FtParams()
        self.L.ftref_params_default(C.byref(p))
        for k, v in kw.items():
            if k == "backend":
                p.backend = v.encode()
            else:
                setattr(p, k, v)
        return p

    def sim_params(self, **kw):
        s = SimParams()
        self.L.ftref_sim_default(C.byref(s))
        for k, v in kw.items():
            setattr(s, k, v)
        return s

    def simulate(self, movers=None, **kw):
        """simulate(); movers: rows of (x_ref, y_ref, vx_pxh, vy_pxh, mag) placed
        instead of the simulation's own random movers."""
        s = self.sim_params(**kw)
        frames = np.empty((s.nframes, s.height, s.width), np.float32)
        mjd = np.empty(s.nframes)
        exp = np.empty(s.nframes)
        mv = _f64(np.asarray(movers if movers is not None else np.zeros((0, 5)), np.float64).reshape(-1, 5))
        if self.L.ftref_simulate_movers(C.byref(s), mv.ravel(), mv.shape[0], frames, mjd, exp):
            raise RuntimeError(self.err())
        return frames, mjd, exp

    def build_stage(self, sub, t_h, fwhm_px, params=None, residual=False):
        sub = _f32(sub)
        n, h, w = sub.shape
        p = params or self.params()
        filt = np.empty_like(sub)
        sky = np.empty((h, w), np.float32)
        mask = np.empty((h, w), np.float32)
        sigma = np.empty(n)
        cr = np.empty(n, np.int32)
        res = np.empty_like(sub) if residual else None
        rc = self.L.ftref_build_stage(sub, n, w, h, _f64(t_h), fwhm_px, C.byref(p), filt, sky, mask, sigma, cr,
                                      None if res is None else res.ctypes.data_as(C.c_void_p))
        if rc:
            raise RuntimeError(self.err())
        out = dict(filtered=filt, static_sky=sky, mask=mask, sigma=sigma, cr=cr)
        if residual:
            out["residual"] = res
        return out

    def stack(self, frames, dx=None, dy=None, t_h=None, vel=None, min_count=3, which=0, threads=0):
        frames = _f32(frames)
        n, h, w = frames.shape
        keep = []

        def ptr(a, conv):
            if a is None:
                return None
            a = conv(a)
            keep.append(a)
            return a.ctypes.data_as(C.c_void_p)
        m = (np.asarray(dx).size // n) if dx is not None else np.asarray(vel).shape[0]
        ms = np.empty((h, w), np.float32)
        bv = np.empty((h, w), np.int32)
        rc = self.L.ftref_stack(frames, w, h, n, ptr(dx, _i32), ptr(dy, _i32), ptr(t_h, _f64), ptr(vel, _f64), m,
                                min_count, threads, which, ms, bv)
        if rc:
            raise RuntimeError(self.err())
        return ms, bv

    def check_backend(self, name):
        """The reference's check-backend procedure for backend `name`:
        (conforming checks, checks, bit-identical checks, report text)."""
        buf = C.create_string_buffer(4096)
        total, same = C.c_int(), C.c_int()
        ok = self.L.ftref_check_backend(name.encode(), buf, 4096, C.byref(total), C.byref(same))
        if ok < 0:
            raise RuntimeError(self.err())
        return ok, total.value, same.value, buf.value.decode()

    def cuda_available(self):
        return bool(self.L.ftref_cuda_available())

    def stack_cuda_timed(self, frames, t_h, vel, min_count):
        """The reference CUDA backend's pass (straight-line shifts) and its own
        timings: dict(max_snr, best_v, upload, kernel, download, setup)."""
        frames = _f32(frames)
        n, h, w = frames.shape
        vel = _f64(vel)
        ms = np.empty((h, w), np.float32)
        bv = np.empty((h, w), np.int32)
        tm = np.zeros(4)
        if self.L.ftref_stack_cuda_timed(frames, w, h, n, _f64(t_h), vel.ravel(), vel.shape[0], min_count, ms, bv, tm):
            raise RuntimeError(self.err())
        return dict(max_snr=ms, best_v=bv, upload=tm[0], kernel=tm[1], download=tm[2], setup=tm[3])

    def velocity_grid(self, span_h, **kw):
        p = self.params(**kw)
        dv = C.c_double()
        cnt = self.L.ftref_velocity_grid(span_h, C.byref(p), None, 0, C.byref(dv))
        out = np.empty((cnt, 2))
        self.L.ftref_velocity_grid(span_h, C.byref(p), out.ctypes.data_as(C.c_void_p), cnt, C.byref(dv))
        return out, dv.value

    def null_orders(self, t_h, runs, seed):
        t_h = _f64(t_h)
        out = np.empty((runs, t_h.size))
        self.L.ftref_null_orders(t_h, t_h.size, runs, seed, out)
        return out

    def find_peaks(self, max_snr, best_v, floor, radius, edge, max_peaks):
        max_snr, best_v = _f32(max_snr), _i32(best_v)
        h, w = max_snr.shape
        cap = max(1, w * h)
        px, py, pv = (np.empty(cap, np.int32) for _ in range(3))
        ps = np.empty(cap, np.float32)
        k = self.L.ftref_find_peaks(max_snr, best_v, w, h, floor, radius, edge, max_peaks, px, py, ps, pv)
        return px[:k], py[:k], ps[:k], pv[:k]

    def set_threshold(self, pooled, runs, **kw):
        pooled = _f32(pooled)
        p = self.params(**kw)
        meth = C.create_string_buffer(32)
        a, k, s2 = C.c_double(), C.c_double(), C.c_double()
        thr = self.L.ftref_set_threshold(pooled, pooled.size, runs, C.byref(p), meth, C.byref(a), C.byref(k),
                                         C.byref(s2))
        return thr, meth.value.decode(), a.value, k.value, s2.value

    def prepare(self, frames, mjd, exptime, reg_dx=None, reg_dy=None, **kw):
        """prepare() (preprocess.cpp:528-585); reg_dx / reg_dy: per-frame
        registration offsets (Frame::reg_dx, types.hpp:61-65) or None."""
        frames = _f32(frames)
        n, h, w = frames.shape
        p = self.params(**kw)
        rx = ry = None
        if reg_dx is not None:
            rx, ry = _f64(reg_dx), _f64(reg_dy)
        hp = self.L.ftref_prepare_reg(n, w, h, frames, _f64(mjd), _f64(exptime),
                                      None if rx is None else rx.ctypes.data_as(C.c_void_p),
                                      None if ry is None else ry.ctypes.data_as(C.c_void_p), C.byref(p))
        if not hp:
            raise RuntimeError(self.err())
        return Prepared(self, hp)

    def load_frames(self, paths):
        """load_frames() (fits.hpp:86) of FITS files: dict(frames, mjd, exptime,
        reg_dx, reg_dy) with reg_dx / reg_dy None unless every frame has them."""
        joined = "\n".join(paths).encode()
        w, h, n, has = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        if self.L.ftref_load_frames(joined, None, None, None, None, None, C.byref(has), C.byref(w), C.byref(h),
                                    C.byref(n)):
            raise RuntimeError(self.err())
        frames = np.empty((n.value, h.value, w.value), np.float32)
        mjd, exp, rx, ry = (np.empty(n.value) for _ in range(4))
        ptr = lambda a: a.ctypes.data_as(C.c_void_p)
        if self.L.ftref_load_frames(joined, ptr(frames), ptr(mjd), ptr(exp), ptr(rx), ptr(ry), C.byref(has),
                                    C.byref(w), C.byref(h), C.byref(n)):
            raise RuntimeError(self.err())
        return dict(frames=frames, mjd=mjd, exptime=exp, reg_dx=rx if has.value else None,
                    reg_dy=ry if has.value else None)

    def completeness(self, frames, mjd, exptime, snr_levels, per_level, min_separation, seed, **kw):
        """The reference's completeness() (validate.cpp:62-165) on raw frames."""
        frames = _f32(frames)
        n, h, w = frames.shape
        lv = _f64(snr_levels)
        rows = np.empty((lv.size, 7))
        thr, s50 = C.c_double(), C.c_double()
        ok = C.c_int()
        meth = C.create_string_buffer(32)
        p = self.params(**kw)
        if self.L.ftref_completeness(n, w, h, frames, _f64(mjd), _f64(exptime), C.byref(p), lv, lv.size, per_level,
                                     C.c_double(min_separation), C.c_ulonglong(seed), rows.ctypes.data_as(C.c_void_p),
                                     C.byref(thr), meth, C.byref(ok), C.byref(s50)):
            raise RuntimeError(self.err())
        keys = ("target_snr", "injected", "recovered", "detected", "mean_snr", "mean_dpos", "mean_dv")
        out = [dict(zip(keys, r)) for r in rows]
        for r in out:
            for k in ("injected", "recovered", "detected"):
                r[k] = int(r[k])
        return dict(rows=out, threshold=thr.value, method=meth.value.decode(), baseline_ok=ok.value, snr50=s50.value)

    def inject(self, frames, mjd, exptime, objects, t_ref_mjd, fwhm_px):
        frames = _f32(frames).copy()
        n, h, w = frames.shape
        obj = _f64(objects).reshape(-1, 5)
        self.L.ftref_inject(frames, n, w, h, _f64(mjd), _f64(exptime), _f64(obj.ravel()), obj.shape[0], t_ref_mjd,
                            fwhm_px)
        return frames

    def iso_from_mjd(self, mjd, decimals):
        buf = C.create_string_buffer(96)
        self.L.ftref_iso_from_mjd(mjd, decimals, buf, 96)
        return buf.value.decode()

    def check_registration(self, frames, t_h):
        """check_registration of frames (n, h, w) at t_h hours, as a dict."""
        frames = _f32(frames)
        n, h, w = frames.shape
        out = np.zeros(9)
        msg = C.create_string_buffer(1024)
        if self.L.ftref_check_registration(frames, n, w, h, _f64(t_h), out, msg, 1024) != 0:
            raise RuntimeError(self.L.ftref_last_error().decode())
        return drift_dict(out, msg.value.decode())


DRIFT_KEYS = ("measured", "registered", "dx", "dy", "mid_dx", "mid_dy", "rate_pxh", "stars", "matched")


def drift_dict(values, message):
    """A DriftCheck as a dict: flags and counts as ints, offsets as floats."""
    d = {k: float(v) for k, v in zip(DRIFT_KEYS, values)}
    for k in ("measured", "registered", "stars", "matched"):
        d[k] = int(d[k])
    d["message"] = message
    return d


class Prepared:
    def __init__(self, ref, hp):
        self.ref, self.hp = ref, hp
        L = ref.L
        w, h, n = C.c_int(), C.c_int(), C.c_int()
        fwhm, span, tref = C.c_double(), C.c_double(), C.c_double()
        L.ftref_prep_info(hp, C.byref(w), C.byref(h), C.byref(n), C.byref(fwhm), C.byref(span), C.byref(tref))
        self.w, self.h, self.n = w.value, h.value, n.value
        self.fwhm, self.span_h, self.t_ref = fwhm.value, span.value, tref.value

    def __del__(self):
        try:
            self.ref.L.ftref_prep_free(self.hp)
        except Exception:
            pass

    def vectors(self):
        n = self.n
        t, s, b = np.empty(n), np.empty(n), np.empty(n)
        cr, rank = np.empty(n, np.int32), np.empty(n, np.int32)
        self.ref.L.ftref_prep_vectors(self.hp, *(a.ctypes.data_as(C.c_void_p) for a in (t, s, b, cr, rank)))
        return dict(t_h=t, sigma=s, background=b, cr=cr, rank=rank)

    def images(self):
        n, h, w = self.n, self.h, self.w
        sub = np.empty((n, h, w), np.float32)
        filt = np.empty((n, h, w), np.float32)
        sky = np.empty((h, w), np.float32)
        mask = np.empty((h, w), np.float32)
        self.ref.L.ftref_prep_images(self.hp, *(a.ctypes.data_as(C.c_void_p) for a in (sub, filt, sky, mask)))
        return dict(sub=sub, filtered=filt, static_sky=sky, mask=mask)

    def is_artefact_peak(self, x, y, snr, vidx, vx, vy, **kw):
        p = self.ref.params(**kw)
        return self.ref.L.ftref_is_artefact_peak(self.hp, x, y, snr, vidx, vx, vy, C.byref(p))

    def with_times(self, t_h, **kw):
        p = self.ref.params(**kw)
        hp = self.ref.L.ftref_with_times(self.hp, _f64(t_h), C.byref(p))
        if not hp:
            raise RuntimeError(self.ref.err())
        return Prepared(self.ref, hp)

    def search(self, csv_path=None, **kw):
        """search() of the prepared sequence; with csv_path, the reference's
        candidate file is written there and returned as candidates_csv."""
        p = self.ref.params(**kw)
        rp = self.ref.L.ftref_search(self.hp, C.byref(p))
        if not rp:
            raise RuntimeError(self.ref.err())
        L = self.ref.L
        t_ref, fwhm = C.c_double(), C.c_double()
        if L.ftref_result_csv(rp, csv_path.encode() if csv_path else None, C.byref(t_ref), C.byref(fwhm)) != 0:
            L.ftref_result_free(rp)
            raise RuntimeError(self.ref.err())
        csv_text = open(csv_path).read() if csv_path else None
        meth = C.create_string_buffer(32)
        dv, a, k, s2 = C.c_double(), C.c_double(), C.c_double(), C.c_double()
        nv, nc, npk = C.c_int(), C.c_int(), C.c_int()
        thr = L.ftref_result_scalars(rp, meth, C.byref(dv), C.byref(nv), C.byref(nc), C.byref(npk), C.byref(a),
                                     C.byref(k), C.byref(s2))
        ms = np.empty((self.h, self.w), np.float32)
        nulls = np.empty(npk.value)
        L.ftref_result_arrays(rp, ms.ctypes.data_as(C.c_void_p), nulls.ctypes.data_as(C.c_void_p))
        cands = []
        for i in range(nc.value):
            v = np.empty(17)
            fl = C.create_string_buffer(64)
            L.ftref_result_candidate(rp, i, v, fl)
            cands.append((v, fl.value.decode()))
        tracks = np.zeros((nc.value, self.n, 5))
        for i in range(nc.value):
            for f in range(self.n):
                L.ftref_track_point(self.hp, rp, i, f, tracks[i, f])
        L.ftref_result_free(rp)
        return dict(threshold=thr, method=meth.value.decode(), dv=dv.value, n_velocities=nv.value,
                    null_peaks=nulls, max_snr=ms, candidates=cands, null_a=a.value, null_k=k.value,
                    null_inv_s2=s2.value, t_ref_mjd=t_ref.value, fwhm=fwhm.value, candidates_csv=csv_text,
                    track_points=tracks)
