// The search around the stacking passes: motion grid, time-shuffled null runs,
// null-peak screening, the tail fit and threshold (FaintTrail search.cpp), with
// the per-pixel work on the device and the small sequential steps on the host.
#pragma once

#include <cstdint>
#include <functional>
#include <map>
#include <memory>
#include <string>
#include <utility>
#include <vector>

#include "engine.h"
#include "stage.h"
#include "candidate.h"
#include "registration.h"

namespace ftb {

// SearchParams fields used by the search path (search.hpp:18-90).
struct SearchParams {
    double vmin_pxh = 4.0, vmax_pxh = 40.0, grid_tol_px = 0.5, fwhm_px = 0.0;
    double clip_sigma = 8.0, cr_sigma = 5.0, mask_scatter = 2.5, weight_scatter = 1.5;
    double min_coverage = 0.7, threshold_snr = 0.0, min_snr_floor = 5.0, target_false_per_run = 0.02;
    double max_frame_fraction = 0.25;
    int static_exclude = -1, null_runs = 3, null_tested = 3000, max_candidates = 300, edge_px = 4;
    bool gauss_model = true;  // null_model "gauss" (else "linear")
    int passes_per_launch = 0;  // 0: as many as fit; k: at most k per launch
    double half_tolerance = 3.0;  // allowed shortfall of each half's S/N (search.hpp:66)
    // null runs split over shard_count calls (one per GPU): this call runs block
    // shard_index of the null runs and, on shard 0 only, the real pass
    int shard_index = 0, shard_count = 1;
    // > 0: the null-run threshold (and its tail fit) is given: no null runs
    double calibrated_threshold = 0.0, cal_a = 0.0, cal_b = 0.0, cal_k = 0.0, cal_inv_s2 = 0.0;
    uint64_t seed = 12345;
    // registration check before the preprocessing (search.hpp:76-81): 0 off,
    // 1 check, 2 auto (check; frames that are not registered are an error, as no
    // alignment is done here)
    int align = 0;
    // registration offsets per frame (detector = registered + offset; the caller's
    // frame order), from the FITS keywords REGDX / REGDY (types.hpp:61-65); empty:
    // none, and the detector test of the artefact screen is off (search.cpp:196-225)
    std::vector<double> reg_dx, reg_dy;
};

struct Peak {
    int x = 0, y = 0;
    float snr = 0.0f;
    int vidx = -1;
};

// xoshiro256** seeded by splitmix64, the reference's Rng (random.hpp:14-38):
// the null-run permutations and the completeness placements draw from it.
class Xoshiro {
public:
    explicit Xoshiro(uint64_t seed) {
        uint64_t z = seed;
        for (auto& v : s_) {
            uint64_t r = (z += 0x9e3779b97f4a7c15ULL);
            r = (r ^ (r >> 30)) * 0xbf58476d1ce4e5b9ULL;
            r = (r ^ (r >> 27)) * 0x94d049bb133111ebULL;
            v = r ^ (r >> 31);
        }
    }
    double uniform() { return static_cast<double>(next() >> 11) * (1.0 / 9007199254740992.0); }
    double uniform(double a, double b) { return a + (b - a) * uniform(); }

private:
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next() {
        const uint64_t out = rotl(s_[1] * 5, 7) * 9;
        const uint64_t t = s_[1] << 17;
        s_[2] ^= s_[0];
        s_[3] ^= s_[1];
        s_[1] ^= s_[2];
        s_[0] ^= s_[3];
        s_[2] ^= t;
        s_[3] = rotl(s_[3], 45);
        return out;
    }
    uint64_t s_[4];
};

// ---- host steps (bit-identical restatements of the reference's host code)
std::vector<std::pair<double, double>> velocity_grid(double span_h, const SearchParams& p, double* dv_out);
std::vector<std::vector<double>> null_time_orders(const std::vector<double>& t_h, int runs, uint64_t seed);
void shift_table(const std::vector<double>& t_h, const std::vector<std::pair<double, double>>& grid,
                 std::vector<int>& dx, std::vector<int>& dy);
int pass_min_count(double min_coverage, int n);
// find_peaks' order: raster-ordered candidates sorted by std::sort on S/N
// descending, then truncated (search.cpp:105-135)
void order_peaks(std::vector<Peak>& raster_ordered, size_t max_peaks);
struct Threshold {
    double snr = 0.0;
    std::string method;
    double a = 0.0, b = 0.0, k = 0.0, inv_s2 = 0.0;
};
// set_threshold with null runs, or fixed (search.cpp:573-598); the Gaussian
// trial-count rule for runs == 0 without a fixed threshold (search.cpp:599-611)
Threshold set_threshold(const SearchParams& p, const std::vector<float>& pooled, int runs, double fwhm_px, int w,
                        int h, size_t n_motions);
double estimate_fwhm(const std::vector<float>& img, int w, int h, double noise_sigma);
double estimate_psf_fwhm(const std::vector<float>& static_sky, int w, int h, std::vector<double> sigma,
                         const SearchParams& p);
double median_of(std::vector<float> v);  // median_inplace (common.hpp:64-74)

// ---- device steps
// prepare_core's background and blank-border growth (preprocess.cpp:572-580,
// 233-254): d_raw (overwritten) -> d_sub; per-frame backgrounds to h_bg.
void prepare_sub(Context& c, StageScratch& sc, float* d_raw, float* d_sub, int w, int h, int n, double* h_bg);
// local maxima of a detection map above `floor` (search.cpp:105-131), in
// raster order
std::vector<Peak> device_peaks(Context& c, const float* d_max, const int* d_best_v, int w, int h, float floor,
                               int radius, int edge);
// The same for many maps at once (the null runs of a batch): every peak kernel
// is queued, one sync brings all candidate lists back, and the host orders them
// (raster order, then order_peaks with `keep`) on a thread per map.
struct PeakMap {
    const float* d_max;
    const int* d_best_v;
};
std::vector<std::vector<Peak>> device_peaks_many(Context& c, const std::vector<PeakMap>& maps, int w, int h,
                                                 float floor, int radius, int edge, size_t keep);
// A null run's peaks as its pooled list needs them (order_peaks with `keep`, then
// the first `tested` screened for artefacts, search.cpp:766-781): the screened
// peaks (in any order) and the S/N values of the ranks after them, down to the
// truncation, in descending order. Equal values are interchangeable in the
// pooled list, so a full sort is needed only when a tie straddles the screening
// boundary (then the reference's std::sort decides which peaks are screened).
struct NullPeaks {
    std::vector<Peak> tested;
    std::vector<float> rest;
};
NullPeaks split_null_peaks(std::vector<Peak> raster_ordered, size_t keep, size_t tested);

// artefact flags (single-frame share, field edge) of the first count[k] peaks of
// every null run k at their grid motions (is_artefact_peak, search.cpp:229-243,
// 142-190), on the device, one sync
struct ArtefactJob {
    const std::vector<Peak>* peaks;
    size_t count;
    const float* d_filtered;
    const float* d_sky;
    const std::vector<double>* t_h;
};
// Rows [oy, oy + rows) of an image whose frames a step holds (rows 0: all).
struct Band {
    int oy = 0, rows = 0;
};
// reg_dx / reg_dy: registration offsets in frame order (empty: no detector test).
// band: the device frames (d_sub and the jobs' filtered frames and sky) hold
// these rows of the w x h image; peaks are in image coordinates.
std::vector<std::vector<char>> device_artefacts_many(Context& c, const std::vector<ArtefactJob>& jobs,
                                                     const std::vector<std::pair<double, double>>& grid,
                                                     const float* d_sub, int w, int h, int n, double fwhm_px,
                                                     double max_frame_fraction, const std::vector<double>& reg_dx,
                                                     const std::vector<double>& reg_dy, Band band = {});

// detector_flag's grid of offsets (search.cpp:217-220): -span, -span + 0.5, ...
// while <= span, each step an addition of 0.5 as the reference's loop makes it,
// span = max(2, 2 fwhm)
std::vector<double> detector_steps(double fwhm_px);

// An object injected into every frame of a copy (Injection, validate.hpp:18-23).
struct Injection {
    double x_ref = 0, y_ref = 0, vx_pxh = 0, vy_pxh = 0, flux = 0;
};

// The pixel increments inject() makes (validate.cpp:17-29 through add_trailed /
// add_gaussian, psf.hpp:20-58), computed on the host with the reference's double
// arithmetic, in the reference's order: one patch per Gaussian, frames in order.
struct InjectionPatches {
    std::vector<int> frame, x0, y0, pw, ph;  // per patch
    std::vector<size_t> off;                 // into values
    std::vector<float> values;               // the float increments, row-major per patch
};
InjectionPatches injection_patches(const std::vector<Injection>& objects, const std::vector<double>& t_mid_h,
                                   const std::vector<double>& exptime_s, double fwhm_px, int w, int h);
// Adds the patches to device frames (n x h x pitch) in order.
void apply_patches(Context& c, const InjectionPatches& ip, float* d_frames, int w, int h, int n);

struct SearchOut {
    int w = 0, h = 0, n = 0;
    double fwhm_px = 0, span_h = 0, t_ref_mjd = 0, dv = 0;
    std::vector<double> t_h, background, sigma;
    std::vector<double> reg_dx, reg_dy;  // registration offsets in time order (empty: none)
    std::vector<std::pair<double, double>> grid;
    Threshold thr;
    std::vector<double> null_peaks;      // pooled S/N of the null runs (search.hpp:177)
    std::vector<Peak> peaks;             // real-run peaks above the floor (find_peaks)
    std::vector<Peak> selected;          // select_peaks (search.cpp:614-620)
    std::vector<float> max_snr;          // real detection map
    std::vector<int> best_v;
    std::vector<Candidate> candidates;   // refined selected peaks (search.cpp:786-804)
    DriftCheck registration;             // the registration check, if one ran (search.hpp:122)
    double adds = 0;                     // pixel x frame x motion additions of all passes
};

// expected_null_peaks (search.cpp:697-702): null peaks per run above `snr`
double expected_null_peaks(const Threshold& t, double snr);

// The device frames a refinement reads: filtered, the real residuals, sub,
// static sky and mask, all with the frame pitch.
struct RefineInputs {
    const float* d_filt;
    const float* d_res;
    const float* d_sub;
    const float* d_sky;
    const float* d_mask;
    int w, h, pitch, n;
    Band band;  // the frames hold these rows of the w x h image (rows 0: all)
};
// refine() of every selected peak and finish_candidates() (search.cpp:245-400,
// 620-676): the candidate list, ordered and numbered as the reference's
std::vector<Candidate> refine_candidates(Context& c, const SearchOut& o, const SearchParams& p, const RefineInputs& in);
// The two halves: refine() of the peaks `keep` (refine_with_contrib, search.cpp:
// 245-397; a band's peaks with that band's frames), then finish_candidates over
// all of them (duplicates, ghosts, flags, false-alarm rates, order, ids).
struct RefinedCandidate {
    Candidate c;
    std::vector<double> contrib;  // per-frame track values
};
std::vector<RefinedCandidate> refine_tracks(Context& c, const SearchOut& o, const SearchParams& p,
                                            const RefineInputs& in, const std::vector<Peak>& keep);
std::vector<Candidate> finish_candidates(const SearchOut& o, std::vector<RefinedCandidate> rc);

// One search request in phases, so that the passes of several searches (or of
// one search's null runs and copies) can be stacked in shared launches:
// prepare (upload, background, the real stage, grid, time orders), stage a range
// of items (null runs first, then injection copies) appending their pass jobs
// (the real pass with the first call), finish those items after the jobs ran
// (peaks, artefact screen, pooling), finalize (threshold, copies' peaks, maps).
class SearchRequest {
public:
    SearchRequest(Context& c, const SearchParams& p, int w, int h, int n);
    void prepare(const float* frames, const double* mjd, const double* exptime, bool on_device, int in_pitch,
                 bool keep_raw, const std::function<void(double, const char*)>& report);
    int runs() const { return runs_; }
    size_t item_bytes() const;                        // device bytes one null run or copy holds in flight
    void expect_copies(bool on) { copies_ = on; }     // copies hold their own frames until their refinement
    static size_t base_bytes(int w, int h, int n);    // device bytes of a prepared request
    // The shift tables of the passes stage_items(k0, k1) queues, in its order
    // (frame and map pointers unset), for planning ahead.
    std::vector<PassJob> pass_tables(int k0, int k1) const;
    // Queues the preprocessing of items [k0, k1) (and the real pass, the first
    // time) and fills the frame and map pointers of jobs[at ..], which hold
    // pass_tables(k0, k1); with at = kAppend the jobs are appended, tables made.
    static constexpr size_t kAppend = ~size_t{0};
    void stage_items(int k0, int k1, const std::vector<std::vector<Injection>>& copies, std::vector<PassJob>& jobs,
                     size_t at = kAppend);
    void finish_items(int k0, int k1);
    SearchOut finalize(std::vector<SearchOut>* copies_out);

private:
    struct Item {
        DevBuf filt, sky, mask, max, bv;
        DevBuf sub, res;  // a copy's own background-subtracted frames and residuals
        std::vector<double> background, sigma;
    };
    PassJob job(const float* frames, const std::vector<double>& t, float* d_max, int* d_bv) const;
    Context& c_;
    SearchParams p_;
    SearchOut o_;
    StageParams sp_;
    int pitch_ = 0;
    size_t plane_ = 0, map_bytes_ = 0, m_ = 0;
    bool auto_thr_ = true, real_queued_ = false, real_done_ = false, raw_needed_ = false;
    int runs_ = 0, runs_total_ = 0, nms_ = 2, edge_ = 1, min_count_ = 3;
    bool real_ = true, sharded_ = false, calibrated_ = false;
    float floor_ = 0;
    std::vector<std::vector<double>> orders_;
    std::vector<double> exp_sorted_;
    std::vector<float> pooled_;
    DevBuf raw_, raw0_, sub_, filt_, sky_, mask_, max_, bv_;
    bool copies_ = false;
    DevBuf res_;  // the real residuals, for the candidates' photometry
    std::unique_ptr<StageScratch> sc_;
    std::map<int, Item> items_;
};

// frames: host (n x h x w) or, with frames_on_device, device rows of in_pitch
// floats (left untouched; copied in time order).
SearchOut search_host(Context& c, const float* frames, int w, int h, int n, const double* mjd, const double* exptime,
                      const SearchParams& p, const Progress& progress, bool frames_on_device = false,
                      int in_pitch = 0);

// The search plus injection-recovery copies (completeness's searches,
// validate.cpp:88-126): each copy is the raw frames with its objects injected,
// prepared again and searched with the threshold the null runs calibrated
// (fixed, no null runs) and the same PSF width. The real pass, the null runs and
// the copies are stacked together in persistent launches. copies_out receives
// one result per copy (peaks above the threshold, selected peaks, maps).
// The injection-recovery test (completeness, validate.cpp:62-165): the
// threshold calibrated once on the data, then per S/N level `per_level` objects
// placed by the seeded generator away from each other and from the objects the
// data already holds, injected, searched with that threshold held fixed (all
// levels' copies in one batch), and matched to the candidates.
struct CompletenessRow {
    double target_snr = 0;
    int injected = 0, recovered = 0, detected = 0;
    double mean_snr = 0, mean_dpos = 0, mean_dv = 0;
};
struct CompletenessOut {
    std::vector<CompletenessRow> rows;
    double threshold_snr = 0;
    std::string threshold_method;
    int baseline_ok = 0;
    double snr50 = 0;
};
CompletenessOut completeness_host(Context& c, const float* frames, int w, int h, int n, const double* mjd,
                                  const double* exptime, const SearchParams& p, const std::vector<double>& levels,
                                  int per_level, double min_separation, uint64_t seed);

// The tiled search (search_tiled, tiled.cpp:272-647) of host frames (n x h x w)
// in full-width bands of band_rows core rows (0: 1024), for sequences larger
// than HBM: the same result as search_host, bit for bit (tiled.cu).
SearchOut search_tiled_host(Context& c, const float* frames, int w, int h, int n, const double* mjd,
                            const double* exptime, const SearchParams& p, int band_rows, const Progress& progress);

SearchOut search_batch_host(Context& c, const float* frames, int w, int h, int n, const double* mjd,
                            const double* exptime, const SearchParams& p,
                            const std::vector<std::vector<Injection>>& copies, std::vector<SearchOut>& copies_out,
                            const Progress& progress, bool frames_on_device = false, int in_pitch = 0);

}  // namespace ftb
