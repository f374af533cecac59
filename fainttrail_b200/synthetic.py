"""Seeded synthetic observing sequences for the benchmark workloads.

Frames follow the benchmark model: a 1000 ADU sky (1 % frame-to-frame level
variation), Gaussian read noise sigma 10 plus photon noise (normal, variance =
sky, as the reference simulator's Poisson deviate is above a mean of 64), static
stars with log-uniform flux and a Gaussian PSF of FWHM 2.5 px, and movers placed
at a target stack S/N with the reference's flux_for_snr rule (validate.cpp:31-34)
and trailed over the exposure. Generated on the device with torch (plumbing;
nothing here is on the measured path). The named workloads carry the search
parameters of their configuration: rates in px/min -> px/h, a half-pixel grid
step over the span (grid_tol_px 0.125).
"""
import math
from dataclasses import dataclass, field

import numpy as np

FWHM_TO_SIGMA = 1.0 / 2.354820045030949


@dataclass
class Workload:
    name: str
    width: int
    height: int
    nframes: int
    cadence_s: float
    exptime_s: float
    nstars: int
    nmovers: int
    snr: tuple
    rate_px_min: tuple
    null_runs: int
    fwhm_px: float = 2.5
    sky_adu: float = 1000.0
    read_noise: float = 10.0
    extra: dict = field(default_factory=dict)

    def search_params(self):
        return dict(vmin_pxh=self.rate_px_min[0] * 60.0, vmax_pxh=self.rate_px_min[1] * 60.0, grid_tol_px=0.125,
                    fwhm_px=self.fwhm_px, null_runs=self.null_runs)

    def times(self):
        mjd0 = 61337.9
        mid = mjd0 + (np.arange(self.nframes) * self.cadence_s + 0.5 * self.exptime_s) / 86400.0
        return mid, np.full(self.nframes, self.exptime_s)


WORKLOADS = {
    # plain CPU-runnable search: 20 x 1024^2, 60 s cadence, 8 null shuffles
    "plain-1k": Workload("plain-1k", 1024, 1024, 20, 60.0, 45.0, 200, 5, (3.0, 8.0), (0.2, 1.1), 8),
    # full-frame plain search on one B200: 40 x 4096^2, 30 s cadence, 3 null shuffles
    "fullframe-4k": Workload("fullframe-4k", 4096, 4096, 40, 30.0, 30.0, 200, 20, (4.0, 10.0), (0.1, 2.0), 3),
    # the full-frame search on a quarter of the area (profiling case; frames still exceed L2)
    "fullframe-2k": Workload("fullframe-2k", 2048, 2048, 40, 30.0, 30.0, 200, 20, (4.0, 10.0), (0.1, 2.0), 3),
    # the full-frame search on 1/16 of the area (ncu captures of the whole-search kernels)
    "fullframe-1k": Workload("fullframe-1k", 1024, 1024, 40, 30.0, 30.0, 50, 5, (4.0, 10.0), (0.1, 2.0), 3),
    # batched null calibration + completeness: 30 x 2048^2, 64 nulls + 16 injection copies
    "batched-2k": Workload("batched-2k", 2048, 2048, 30, 60.0, 45.0, 200, 0, (2.0, 8.0), (0.2, 1.1), 64,
                           extra=dict(injection_copies=16, injected_movers=50)),
    # large-sensor: 60 x 9576 x 6388, 30 s cadence, 32 null shuffles
    "large-sensor": Workload("large-sensor", 9576, 6388, 60, 30.0, 30.0, 1200, 240, (4.0, 10.0), (0.05, 3.0), 32),
}


def flux_for_snr(snr, sigma, fwhm_px, nframes):
    s = fwhm_px * FWHM_TO_SIGMA
    return snr / math.sqrt(max(1, nframes)) * sigma * math.sqrt(4.0 * math.pi) * s


def _add_gauss(img, x0, y0, flux, sigma, torch):
    h, w = img.shape[-2:]
    r = int(math.ceil(4 * sigma)) + 1
    xc, yc = int(math.floor(x0 + 0.5)), int(math.floor(y0 + 0.5))
    xa, xb = max(0, xc - r), min(w - 1, xc + r)
    ya, yb = max(0, yc - r), min(h - 1, yc + r)
    if xa > xb or ya > yb:
        return
    xs = torch.arange(xa, xb + 1, device=img.device, dtype=torch.float64) - x0
    ys = torch.arange(ya, yb + 1, device=img.device, dtype=torch.float64) - y0
    g = torch.exp(-0.5 * (ys[:, None] ** 2 + xs[None, :] ** 2) / sigma ** 2) * (flux / (2 * math.pi * sigma ** 2))
    img[..., ya:yb + 1, xa:xb + 1] += g.to(img.dtype)


def generate(wl, seed=7, device="cuda"):
    """frames (n, h, w) float32 torch tensor on `device`, mjd, exptime, truth."""
    import torch
    rng = np.random.default_rng(seed)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    n, h, w = wl.nframes, wl.height, wl.width
    sigma = wl.fwhm_px * FWHM_TO_SIGMA
    mjd, exptime = wl.times()
    t_ref = 0.5 * (mjd[0] + mjd[-1])
    t_h = (mjd - t_ref) * 24.0
    stars = torch.zeros((h, w), dtype=torch.float32, device=device)
    for _ in range(wl.nstars):
        flux = math.exp(rng.uniform(math.log(2e3), math.log(2e6)))
        _add_gauss(stars, rng.uniform(-5, w + 5), rng.uniform(-5, h + 5), flux, sigma, torch)
    pix_sigma = math.sqrt(wl.sky_adu + wl.read_noise ** 2)
    truth = []
    for _ in range(wl.nmovers):
        snr = rng.uniform(*wl.snr)
        rate = rng.uniform(*wl.rate_px_min) * 60.0
        pa = rng.uniform(0, 2 * math.pi)
        truth.append(dict(x=rng.uniform(24, w - 24), y=rng.uniform(24, h - 24), vx=rate * math.cos(pa),
                          vy=rate * math.sin(pa), snr=snr, flux=flux_for_snr(snr, pix_sigma, wl.fwhm_px, n)))
    frames = torch.empty((n, h, w), dtype=torch.float32, device=device)
    half = 0.5 * wl.exptime_s / 3600.0
    for i in range(n):
        level = wl.sky_adu * (1.0 + 0.01 * float(rng.standard_normal()))
        f = frames[i]
        torch.randn((h, w), generator=gen, device=device, out=f)
        f.mul_(pix_sigma).add_(level).add_(stars)
        for m in truth:
            steps = 4
            for k in range(steps):
                t = t_h[i] - half + (k + 0.5) / steps * 2 * half
                _add_gauss(f, m["x"] + m["vx"] * t, m["y"] + m["vy"] * t, m["flux"] / steps, sigma, torch)
    return frames, mjd, exptime, truth


def injection_copies(wl, frames_shape, seed=11):
    """The injection-recovery copies of a batched workload: `injection_copies`
    sets of `injected_movers` objects (x_ref, y_ref, vx_pxh, vy_pxh, flux) at a
    stack S/N drawn from wl.snr, rates from wl.rate_px_min, uniform PA, placed
    24 px inside the frame, flux by the flux_for_snr rule."""
    n, h, w = frames_shape
    rng = np.random.default_rng(seed)
    pix_sigma = math.sqrt(wl.sky_adu + wl.read_noise ** 2)
    copies = []
    for _ in range(int(wl.extra.get("injection_copies", 0))):
        objs = []
        for _ in range(int(wl.extra.get("injected_movers", 0))):
            snr = rng.uniform(*wl.snr)
            rate = rng.uniform(*wl.rate_px_min) * 60.0
            pa = rng.uniform(0, 2 * math.pi)
            objs.append((rng.uniform(24, w - 24), rng.uniform(24, h - 24), rate * math.cos(pa), rate * math.sin(pa),
                         flux_for_snr(snr, pix_sigma, wl.fwhm_px, n)))
        copies.append(objs)
    return copies


def motion_count(span_h, vmin_pxh, vmax_pxh, grid_tol_px):
    """Trial motions of the square velocity lattice inside the annulus (the
    velocity_grid rule, counted exactly)."""
    dv = 4.0 * max(0.05, grid_tol_px) / span_h
    k = int(math.ceil(vmax_pxh / dv))
    lo, hi = max(0.0, vmin_pxh - 0.5 * dv), vmax_pxh + 0.5 * dv
    i = np.arange(-k, k + 1) * dv
    v = np.hypot(i[None, :], i[:, None])
    return int(np.count_nonzero((v >= lo) & (v <= hi)))


def serving_requests(count=16, rate_per_s=20.0, seed=2024, max_adds=5.0e13):
    """A seeded stream of search requests drawn from the serving configuration:
    Poisson arrivals at rate_per_s; frame counts 8-120, widths 512-6000 and
    heights 512-4000 (multiples of 16), a rate range [lo, hi] inside 0.1-3
    px/min, 8-32 null runs; 30 s cadence and the half-pixel motion grid of the
    other configurations. Draws whose work (motions x frames x pixels x passes)
    exceeds max_adds are drawn again (max_adds None keeps every draw): the
    unbounded mix has a median of about 2e14 and a tail to 2e16 adds per request,
    over a thousand times what one GPU serves at 20 requests per second. Returns
    ([(arrival_s, Workload)], draws made)."""
    rng = np.random.default_rng(seed)
    out, t, draws = [], 0.0, 0
    while len(out) < count:
        n = int(rng.integers(8, 121))
        w = int(rng.integers(512, 6001)) // 16 * 16
        h = int(rng.integers(512, 4001)) // 16 * 16
        lo = float(rng.uniform(0.1, 2.5))
        hi = float(rng.uniform(lo + 0.2, 3.0))
        runs = int(rng.integers(8, 33))
        draws += 1
        span_h = (n - 1) * 30.0 / 3600.0
        m = motion_count(span_h, lo * 60.0, hi * 60.0, 0.125)
        if max_adds is not None and float(m) * n * w * h * (1 + runs) > max_adds:
            continue
        t += float(rng.exponential(1.0 / rate_per_s))
        k = len(out)
        out.append((t, Workload(f"serve-{k}", w, h, n, 30.0, 30.0, max(20, w * h // 20000), 3, (5.0, 10.0),
                                (lo, hi), runs)))
    return out, draws
