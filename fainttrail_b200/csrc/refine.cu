// Candidate refinement: FaintTrail's refine() and finish_candidates()
// (search.cpp:245-400, 620-676) for the peaks a search selects. Every sub-pixel
// track S/N (track_snr, search.cpp:142-163) is evaluated on the device, for all
// candidates at once: the two levels of the local (velocity, position) grid,
// the parabola steps, the half-sequence S/N and the per-frame track values; the
// photometry cutout (stack_cutout, search.cpp:826-857) and the field-edge test
// (edge_flag, search.cpp:167-190) are device kernels too. The host replays the
// reference's control flow on the returned values: the strict ">" scan over the
// grid in its loop order, the parabola updates, the flags, the duplicate and
// ghost test, and the final ordering. Sums run in frame order with
// round-to-nearest operations, so every value equals the reference's.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "search.h"
#include "track.cuh"

namespace ftb {

namespace {

constexpr double kFwhmToSigma = 1.0 / 2.354820045030949;  // psf.hpp:16
constexpr double kPi = 3.14159265358979323846;

struct TrackQuery {
    double x, y, vx, vy;
    int which;  // 0: all frames, 1: t < 0, 2: t >= 0
    int pad;
};

struct RefineDev {
    const float* filt;
    const float* res;
    const float* sub;
    const float* sky;
    const float* mask;
    const double* t;
    size_t plane;
    int w, h, pitch, n;
    int oy, rows;  // the frames hold rows [oy, oy + rows) of the w x h image
};

// one query per thread: the S/N of a straight track, optionally with the
// per-frame values and whether the track's pixel is masked in each frame
__global__ void track_eval_kernel(const TrackQuery* q, int nq, RefineDev d, double* snr, float* per_frame,
                                  unsigned char* masked) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nq) return;
    const TrackQuery Q = q[k];
    double sum = 0.0;
    int count = 0;
    for (int i = 0; i < d.n; ++i) {
        const double t = d.t[i];
        if (Q.which == 1 && t >= 0.0) continue;
        if (Q.which == 2 && t < 0.0) continue;
        const double px = track_coord(Q.x, Q.vx, t), py = track_coord(Q.y, Q.vy, t);
        const float v = track_bilinear_band(d.filt + i * d.plane, d.w, d.h, d.pitch, d.oy, d.rows, px, py);
        if (per_frame) {
            per_frame[static_cast<size_t>(k) * d.n + i] = isfinite(v) ? v : CUDART_NAN_F;
            const int xi = static_cast<int>(lround(px)), yi = static_cast<int>(lround(py));
            masked[static_cast<size_t>(k) * d.n + i] =
                xi >= 0 && yi >= 0 && xi < d.w && yi < d.h && yi - d.oy >= 0 && yi - d.oy < d.rows &&
                d.mask[static_cast<size_t>(yi - d.oy) * d.pitch + xi] == 0.0f;
        }
        if (!isfinite(v)) continue;
        sum = __dadd_rn(sum, static_cast<double>(v));
        ++count;
    }
    snr[k] = count >= 3 ? __ddiv_rn(sum, __dsqrt_rn(static_cast<double>(count))) : 0.0;
}

// the mean residual stack along a track on a (2 half + 1)^2 grid: one thread per
// (candidate, pixel), float sums in frame order, then / count
__global__ void cutout_kernel(const double4* track, int K, int half, RefineDev d, float* out) {
    const int size = 2 * half + 1;
    const long long idx = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= static_cast<long long>(K) * size * size) return;
    const int k = static_cast<int>(idx / (size * size)), rem = static_cast<int>(idx % (size * size));
    const int v = rem / size, u = rem % size;
    const double4 tr = track[k];
    float acc = 0.0f;
    int cnt = 0;
    for (int i = 0; i < d.n; ++i) {
        const double cx = track_coord(tr.x, tr.z, d.t[i]), cy = track_coord(tr.y, tr.w, d.t[i]);
        const double sx = __dsub_rn(__dadd_rn(cx, static_cast<double>(u)), static_cast<double>(half));
        const double sy = __dsub_rn(__dadd_rn(cy, static_cast<double>(v)), static_cast<double>(half));
        const float s = track_bilinear_band(d.res + i * d.plane, d.w, d.h, d.pitch, d.oy, d.rows, sx, sy);
        if (!isfinite(s)) continue;
        acc = __fadd_rn(acc, s);
        ++cnt;
    }
    out[idx] = cnt == 0 ? CUDART_NAN_F : __fdiv_rn(acc, static_cast<float>(cnt));
}

// detector_flag (search.cpp:196-225): one warp per candidate, the largest S/N
// of a source fixed on the detector near the track (track.cuh)
__global__ void detector_kernel(const double4* track, int K, RefineDev d, const double* reg, const double* steps,
                                int nsteps, double* best) {
    const int k = static_cast<int>((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (k >= K) return;  // the whole warp
    const double4 t = track[k];
    const double b = detector_best_fixed(d.filt, d.plane, d.w, d.h, d.pitch, d.oy, d.rows, d.n, d.t, reg, reg + d.n,
                                         steps, nsteps, t.x, t.y, t.z, t.w);
    if ((threadIdx.x & 31) == 0) best[k] = b;
}

// field edge: frames whose track pixel has a blank (non-finite sub or static
// sky, or outside) pixel within r; one thread per (candidate, frame)
__global__ void edge_kernel(const double4* track, int K, int r, RefineDev d, int* near_blank) {
    const long long idx = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= static_cast<long long>(K) * d.n) return;
    const int k = static_cast<int>(idx / d.n), i = static_cast<int>(idx % d.n);
    const double4 tr = track[k];
    const int xi = static_cast<int>(lround(track_coord(tr.x, tr.z, d.t[i])));
    const int yi = static_cast<int>(lround(track_coord(tr.y, tr.w, d.t[i])));
    for (int dy = -r; dy <= r; ++dy)
        for (int dx = -r; dx <= r; ++dx) {
            const int xx = xi + dx, yy = yi + dy;
            if (xx < 0 || yy < 0 || xx >= d.w || yy >= d.h || yy - d.oy < 0 || yy - d.oy >= d.rows ||
                !isfinite(d.sub[i * d.plane + static_cast<size_t>(yy - d.oy) * d.pitch + xx]) ||
                !isfinite(d.sky[static_cast<size_t>(yy - d.oy) * d.pitch + xx])) {
                atomicAdd(near_blank + k, 1);
                return;
            }
        }
}

struct TrackState {
    double bx, by, bvx, bvy, best;
};

// add_flag (search.cpp:415-418)
void add_flag(Candidate& c, const std::string& f) {
    if (c.flags.find(f) != std::string::npos) return;
    c.flags += c.flags.empty() ? f : "," + f;
}

bool rejecting(const std::string& f) {  // is_rejecting (search.cpp:398-400)
    return f == "half" || f == "single" || f == "ghost" || f == "edge" || f == "detector";
}

void finalise_flags(Candidate& c) {  // search.cpp:403-413
    c.ok = true;
    size_t start = 0;
    while (start <= c.flags.size() && !c.flags.empty()) {
        const size_t end = c.flags.find(',', start);
        if (rejecting(c.flags.substr(start, end == std::string::npos ? std::string::npos : end - start))) c.ok = false;
        if (end == std::string::npos) break;
        start = end + 1;
    }
}

}  // namespace

std::vector<RefinedCandidate> refine_tracks(Context& c, const SearchOut& o, const SearchParams& p,
                                            const RefineInputs& in, const std::vector<Peak>& keep) {
    const int K = static_cast<int>(keep.size());
    std::vector<RefinedCandidate> rc(static_cast<size_t>(K));
    if (K == 0) return rc;
    const int n = in.n;
    cudaStream_t s = c.stream();
    const double dv = o.dv;
    auto align = [](size_t b) { return (b + 255) / 256 * 256; };
    const int rows = in.band.rows > 0 ? in.band.rows : in.h;
    RefineDev d{in.d_filt, in.d_res, in.d_sub, in.d_sky, in.d_mask, nullptr, static_cast<size_t>(in.pitch) * rows,
                in.w, in.h, in.pitch, n, in.band.oy, rows};

    // the device times, then batches of track queries
    DevBuf& tb = c.scratch(24, align(sizeof(double) * n), "refine times");
    FTB_CHECK(cudaMemcpyAsync(tb.as<double>(), o.t_h.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s));
    d.t = tb.as<double>();
    auto evaluate = [&](const std::vector<TrackQuery>& qs, std::vector<float>* per_frame,
                        std::vector<unsigned char>* masked) {
        const size_t nq = qs.size();
        const size_t qb = align(sizeof(TrackQuery) * nq), sb = align(sizeof(double) * nq);
        const size_t pb = per_frame ? align(sizeof(float) * nq * n) : 0, mb = per_frame ? align(nq * n) : 0;
        DevBuf& buf = c.scratch(25, qb + sb + pb + mb, "refine queries");
        unsigned char* base = buf.as<unsigned char>();
        FTB_CHECK(cudaMemcpyAsync(base, qs.data(), sizeof(TrackQuery) * nq, cudaMemcpyHostToDevice, s));
        double* d_snr = reinterpret_cast<double*>(base + qb);
        float* d_pf = per_frame ? reinterpret_cast<float*>(base + qb + sb) : nullptr;
        unsigned char* d_m = per_frame ? base + qb + sb + pb : nullptr;
        track_eval_kernel<<<static_cast<unsigned>((nq + 127) / 128), 128, 0, s>>>(
            reinterpret_cast<const TrackQuery*>(base), static_cast<int>(nq), d, d_snr, d_pf, d_m);
        FTB_CHECK(cudaGetLastError());
        ++c.launches;
        std::vector<double> snr(nq);
        FTB_CHECK(cudaMemcpyAsync(snr.data(), d_snr, sizeof(double) * nq, cudaMemcpyDeviceToHost, s));
        if (per_frame) {
            per_frame->resize(nq * n);
            masked->resize(nq * n);
            FTB_CHECK(cudaMemcpyAsync(per_frame->data(), d_pf, sizeof(float) * nq * n, cudaMemcpyDeviceToHost, s));
            FTB_CHECK(cudaMemcpyAsync(masked->data(), d_m, nq * n, cudaMemcpyDeviceToHost, s));
        }
        FTB_CHECK(cudaStreamSynchronize(s));
        return snr;
    };

    // start: the peak's pixel and grid motion (search.cpp:248-254)
    std::vector<TrackState> st(static_cast<size_t>(K));
    for (int k = 0; k < K; ++k) {
        const Peak& pk = keep[static_cast<size_t>(k)];
        const auto& v0 = o.grid[static_cast<size_t>(pk.vidx)];
        st[static_cast<size_t>(k)] = {static_cast<double>(pk.x), static_cast<double>(pk.y), v0.first, v0.second, 0.0};
    }
    // two-level local search (search.cpp:256-274): (velocity step, velocity
    // half-range, position step, position half-range); the grid's S/N values come
    // from the device, the strict ">" scan in the reference's loop order here. The
    // first level's centre point is the starting S/N (a + 0 and x + 0 are exact).
    const double levels[2][4] = {{dv / 4, dv, 0.5, 1.0}, {dv / 8, dv / 4, 0.25, 0.5}};
    for (int lv = 0; lv < 2; ++lv) {
        const double* L = levels[lv];
        const int nvs = static_cast<int>(std::lround(L[1] / L[0]));
        const int nps = static_cast<int>(std::lround(L[3] / L[2]));
        const int per = (2 * nvs + 1) * (2 * nvs + 1) * (2 * nps + 1) * (2 * nps + 1);
        std::vector<TrackQuery> qs;
        qs.reserve(static_cast<size_t>(per) * K);
        for (int k = 0; k < K; ++k) {
            const TrackState& t = st[static_cast<size_t>(k)];
            for (int a = -nvs; a <= nvs; ++a)
                for (int b = -nvs; b <= nvs; ++b)
                    for (int i = -nps; i <= nps; ++i)
                        for (int j = -nps; j <= nps; ++j)
                            qs.push_back({t.bx + i * L[2], t.by + j * L[2], t.bvx + a * L[0], t.bvy + b * L[0], 0, 0});
        }
        const std::vector<double> v = evaluate(qs, nullptr, nullptr);
        for (int k = 0; k < K; ++k) {
            TrackState& t = st[static_cast<size_t>(k)];
            const size_t q0 = static_cast<size_t>(k) * per;
            if (lv == 0) {
                const size_t centre = static_cast<size_t>(
                    ((nvs * (2 * nvs + 1) + nvs) * (2 * nps + 1) + nps) * (2 * nps + 1) + nps);
                t.best = v[q0 + centre];
            }
            for (int e = 0; e < per; ++e)
                if (v[q0 + e] > t.best) {
                    t.best = v[q0 + e];
                    const TrackQuery& q = qs[q0 + e];
                    t.bx = q.x;
                    t.by = q.y;
                    t.bvx = q.vx;
                    t.bvy = q.vy;
                }
        }
    }
    // sub-pixel position from a parabola through three samples per axis (:287-297)
    {
        const double hh = 0.25;
        std::vector<TrackQuery> qs;
        for (const TrackState& t : st) {
            qs.push_back({t.bx - hh, t.by, t.bvx, t.bvy, 0, 0});
            qs.push_back({t.bx + hh, t.by, t.bvx, t.bvy, 0, 0});
            qs.push_back({t.bx, t.by - hh, t.bvx, t.bvy, 0, 0});
            qs.push_back({t.bx, t.by + hh, t.bvx, t.bvy, 0, 0});
        }
        const std::vector<double> v = evaluate(qs, nullptr, nullptr);
        for (int k = 0; k < K; ++k) {
            TrackState& t = st[static_cast<size_t>(k)];
            const double sx0 = v[4 * k], sx2 = v[4 * k + 1], sy0 = v[4 * k + 2], sy2 = v[4 * k + 3];
            const double denx = sx0 - 2 * t.best + sx2, deny = sy0 - 2 * t.best + sy2;
            if (denx < 0) t.bx += std::clamp(0.5 * hh * (sx0 - sx2) / denx, -hh, hh);
            if (deny < 0) t.by += std::clamp(0.5 * hh * (sy0 - sy2) / deny, -hh, hh);
        }
    }
    // sub-step motion from a parabola as well (:300-309)
    {
        const double hh = dv / 8;
        std::vector<TrackQuery> qs;
        for (const TrackState& t : st) {
            qs.push_back({t.bx, t.by, t.bvx - hh, t.bvy, 0, 0});
            qs.push_back({t.bx, t.by, t.bvx + hh, t.bvy, 0, 0});
            qs.push_back({t.bx, t.by, t.bvx, t.bvy - hh, 0, 0});
            qs.push_back({t.bx, t.by, t.bvx, t.bvy + hh, 0, 0});
            qs.push_back({t.bx, t.by, t.bvx, t.bvy, 0, 0});
        }
        const std::vector<double> v = evaluate(qs, nullptr, nullptr);
        for (int k = 0; k < K; ++k) {
            TrackState& t = st[static_cast<size_t>(k)];
            const double s0 = v[5 * k], s2 = v[5 * k + 1], t0 = v[5 * k + 2], t2 = v[5 * k + 3], sc = v[5 * k + 4];
            const double denx = s0 - 2 * sc + s2, deny = t0 - 2 * sc + t2;
            if (denx < 0) t.bvx += std::clamp(0.5 * hh * (s0 - s2) / denx, -hh, hh);
            if (deny < 0) t.bvy += std::clamp(0.5 * hh * (t0 - t2) / deny, -hh, hh);
        }
    }
    // the final track: all frames with per-frame values and masks, then the halves
    std::vector<float> per_frame;
    std::vector<unsigned char> masked;
    std::vector<double> all, halves;
    {
        std::vector<TrackQuery> qs;
        for (const TrackState& t : st) qs.push_back({t.bx, t.by, t.bvx, t.bvy, 0, 0});
        all = evaluate(qs, &per_frame, &masked);
        qs.clear();
        for (const TrackState& t : st) {
            qs.push_back({t.bx, t.by, t.bvx, t.bvy, 1, 0});
            qs.push_back({t.bx, t.by, t.bvx, t.bvy, 2, 0});
        }
        halves = evaluate(qs, nullptr, nullptr);
    }
    // photometry cutouts and the edge test
    const double s_psf = o.fwhm_px * kFwhmToSigma;
    const int half = static_cast<int>(std::ceil(3.0 * s_psf));
    const int size = 2 * half + 1;
    const int r_edge = static_cast<int>(std::ceil(2.0 * o.fwhm_px)) + 1;
    std::vector<float> cut(static_cast<size_t>(K) * size * size);
    std::vector<int> near_blank(static_cast<size_t>(K), 0);
    // with registration offsets, the detector test's best fixed-position S/N
    const bool reg = static_cast<int>(o.reg_dx.size()) == n && static_cast<int>(o.reg_dy.size()) == n;
    const std::vector<double> steps = reg ? detector_steps(o.fwhm_px) : std::vector<double>();
    std::vector<double> best_fixed(static_cast<size_t>(K), 0.0);
    {
        const size_t trb = align(sizeof(double4) * K), cb = align(sizeof(float) * cut.size()), eb = align(sizeof(int) * K);
        const size_t rb = reg ? align(sizeof(double) * (2 * static_cast<size_t>(n) + steps.size())) : 0;
        const size_t bb = reg ? align(sizeof(double) * K) : 0;
        DevBuf& buf = c.scratch(26, trb + cb + eb + rb + bb, "refine cutouts");
        unsigned char* base = buf.as<unsigned char>();
        std::vector<double4> tr(static_cast<size_t>(K));
        for (int k = 0; k < K; ++k) {
            const TrackState& t = st[static_cast<size_t>(k)];
            tr[static_cast<size_t>(k)] = make_double4(t.bx, t.by, t.bvx, t.bvy);
        }
        const double4* d_tr = reinterpret_cast<const double4*>(base);
        float* d_cut = reinterpret_cast<float*>(base + trb);
        int* d_nb = reinterpret_cast<int*>(base + trb + cb);
        FTB_CHECK(cudaMemcpyAsync(base, tr.data(), sizeof(double4) * K, cudaMemcpyHostToDevice, s));
        FTB_CHECK(cudaMemsetAsync(d_nb, 0, sizeof(int) * K, s));
        const long long ncut = static_cast<long long>(cut.size());
        cutout_kernel<<<static_cast<unsigned>((ncut + 127) / 128), 128, 0, s>>>(d_tr, K, half, d, d_cut);
        FTB_CHECK(cudaGetLastError());
        ++c.launches;
        const long long nedge = static_cast<long long>(K) * n;
        edge_kernel<<<static_cast<unsigned>((nedge + 127) / 128), 128, 0, s>>>(d_tr, K, r_edge, d, d_nb);
        FTB_CHECK(cudaGetLastError());
        ++c.launches;
        if (reg) {
            std::vector<double> rv(o.reg_dx);
            rv.insert(rv.end(), o.reg_dy.begin(), o.reg_dy.end());
            rv.insert(rv.end(), steps.begin(), steps.end());
            double* d_reg = reinterpret_cast<double*>(base + trb + cb + eb);
            double* d_best = reinterpret_cast<double*>(base + trb + cb + eb + rb);
            FTB_CHECK(cudaMemcpyAsync(d_reg, rv.data(), sizeof(double) * rv.size(), cudaMemcpyHostToDevice, s));
            const long long threads = 32LL * K;
            detector_kernel<<<static_cast<unsigned>((threads + 127) / 128), 128, 0, s>>>(
                d_tr, K, d, d_reg, d_reg + 2 * n, static_cast<int>(steps.size()), d_best);
            FTB_CHECK(cudaGetLastError());
            ++c.launches;
            FTB_CHECK(cudaMemcpyAsync(best_fixed.data(), d_best, sizeof(double) * K, cudaMemcpyDeviceToHost, s));
        }
        FTB_CHECK(cudaMemcpyAsync(cut.data(), d_cut, sizeof(float) * cut.size(), cudaMemcpyDeviceToHost, s));
        FTB_CHECK(cudaMemcpyAsync(near_blank.data(), d_nb, sizeof(int) * K, cudaMemcpyDeviceToHost, s));
        FTB_CHECK(cudaStreamSynchronize(s));
    }

    // the candidates (search.cpp:317-395)
    double t2 = 0.0;
    for (double t : o.t_h) t2 += t * t;
    t2 /= std::max(1, n);
    for (int k = 0; k < K; ++k) {
        const TrackState& t = st[static_cast<size_t>(k)];
        Candidate& cd = rc[static_cast<size_t>(k)].c;
        std::vector<double>& contrib = rc[static_cast<size_t>(k)].contrib;
        cd.snr_coarse = keep[static_cast<size_t>(k)].snr;
        cd.x = t.bx;
        cd.y = t.by;
        cd.vx_pxh = t.bvx;
        cd.vy_pxh = t.bvy;
        cd.snr = all[static_cast<size_t>(k)];
        constexpr double kEmpirical = 1.25;  // the reference's centroid-precision factor
        cd.pos_err_px = cd.snr > 0.0 ? kEmpirical * std::sqrt(2.0) * s_psf / cd.snr : 0.0;
        cd.vel_err_pxh = t2 > 0.0 ? cd.pos_err_px / std::sqrt(t2) : 0.0;
        cd.snr_half1 = halves[2 * static_cast<size_t>(k)];
        cd.snr_half2 = halves[2 * static_cast<size_t>(k) + 1];
        contrib.resize(static_cast<size_t>(n));
        double pos_sum = 0.0, maxc = 0.0;
        int nmasked = 0, inside = 0;
        for (int i = 0; i < n; ++i) {
            const float vf = per_frame[static_cast<size_t>(k) * n + i];
            contrib[static_cast<size_t>(i)] = std::isfinite(vf) ? static_cast<double>(vf) : NAN;
            const double v = contrib[static_cast<size_t>(i)];
            if (!std::isfinite(v)) continue;
            ++inside;
            pos_sum += std::max(0.0, v);
            maxc = std::max(maxc, v);
            if (masked[static_cast<size_t>(k) * n + i]) ++nmasked;
        }
        cd.max_frame_fraction = pos_sum > 0.0 ? maxc / pos_sum : 1.0;
        // PSF photometry on the stacked residuals
        double num = 0.0, den = 0.0;
        const float* ct = cut.data() + static_cast<size_t>(k) * size * size;
        for (int y = 0; y < size; ++y)
            for (int x = 0; x < size; ++x) {
                const float v = ct[static_cast<size_t>(y) * size + x];
                if (!std::isfinite(v)) continue;
                const double kk = std::exp(-0.5 * ((x - half) * (x - half) + (y - half) * (y - half)) / (s_psf * s_psf));
                num += v * kk;
                den += kk * kk;
            }
        cd.flux = den > 0.0 ? num / den * 2.0 * kPi * s_psf * s_psf : 0.0;
        cd.mag_inst = cd.flux > 0.0 ? 25.0 - 2.5 * std::log10(cd.flux) : 99.0;
        // flags
        std::vector<std::string> flags;
        const double expect_half = cd.snr_coarse / std::sqrt(2.0);
        const double half_min = std::max(2.0, expect_half - p.half_tolerance);
        if (cd.snr_half1 < half_min || cd.snr_half2 < half_min) flags.push_back("half");
        if (n >= 8 && cd.max_frame_fraction > p.max_frame_fraction) flags.push_back("single");
        if (inside > 0 && nmasked > inside / 2) flags.push_back("masked");
        if (n > 0 && near_blank[static_cast<size_t>(k)] > std::max(1, n / 10)) flags.push_back("edge");
        if (reg && best_fixed[static_cast<size_t>(k)] >= 0.8 * cd.snr) flags.push_back("detector");
        if (std::hypot(t.bvx, t.bvy) > p.vmax_pxh - 0.5 * dv) flags.push_back("vedge");
        if (std::hypot(t.bvx, t.bvy) < 2.0 * o.fwhm_px / o.span_h) flags.push_back("slow");
        for (size_t i = 0; i < flags.size(); ++i) cd.flags += (i ? "," : "") + flags[i];
    }
    return rc;
}

std::vector<Candidate> finish_candidates(const SearchOut& o, std::vector<RefinedCandidate> rc) {
    const int n = o.n;
    std::vector<Candidate> out;
    // duplicates and ghosts, flags, false-alarm rates, order, ids (:620-676)
    std::sort(rc.begin(), rc.end(),
              [](const RefinedCandidate& a, const RefinedCandidate& b) { return a.c.snr > b.c.snr; });
    const double r_overlap = 1.5 * o.fwhm_px;
    std::vector<bool> drop(rc.size(), false);
    auto pos = [&](const Candidate& cd, int f, double& x, double& y) {
        const double t = o.t_h[static_cast<size_t>(f)];
        x = cd.x + cd.vx_pxh * t;
        y = cd.y + cd.vy_pxh * t;
    };
    for (size_t j = 0; j < rc.size(); ++j) {
        double total = 0.0;
        for (double v : rc[j].contrib)
            if (std::isfinite(v) && v > 0.0) total += v;
        std::vector<bool> shared(static_cast<size_t>(n), false);
        int overlap_max = 0;
        for (size_t i = 0; i < j && !drop[j]; ++i) {
            if (drop[i]) continue;
            int overlap = 0;
            for (int f = 0; f < n; ++f) {
                double xi, yi, xj, yj;
                pos(rc[i].c, f, xi, yi);
                pos(rc[j].c, f, xj, yj);
                const double dx = xi - xj, dy = yi - yj;
                if (dx * dx + dy * dy < r_overlap * r_overlap) {
                    ++overlap;
                    shared[static_cast<size_t>(f)] = true;
                }
            }
            overlap_max = std::max(overlap_max, overlap);
            if (overlap >= n / 2) drop[j] = true;
        }
        if (drop[j] || overlap_max == 0) continue;
        double from_shared = 0.0;
        for (int f = 0; f < n; ++f) {
            const double v = rc[j].contrib[static_cast<size_t>(f)];
            if (shared[static_cast<size_t>(f)] && std::isfinite(v) && v > 0.0) from_shared += v;
        }
        if (total > 0.0 && from_shared / total > 0.3) add_flag(rc[j].c, "ghost");
    }
    for (size_t j = 0; j < rc.size(); ++j) {
        if (drop[j]) continue;
        Candidate cd = rc[j].c;
        finalise_flags(cd);
        cd.false_alarms_per_run = expected_null_peaks(o.thr, cd.snr_coarse);
        out.push_back(cd);
    }
    std::stable_sort(out.begin(), out.end(), [](const Candidate& a, const Candidate& b) {
        if (a.ok != b.ok) return a.ok;
        return a.snr > b.snr;
    });
    for (size_t i = 0; i < out.size(); ++i) out[i].id = static_cast<int>(i + 1);
    return out;
}

std::vector<Candidate> refine_candidates(Context& c, const SearchOut& o, const SearchParams& p, const RefineInputs& in) {
    return finish_candidates(o, refine_tracks(c, o, p, in, o.selected));
}

}  // namespace ftb
