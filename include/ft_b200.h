/* FaintTrail B200 search backend: plain C ABI.
 *
 * A drop-in for the stacking backend and the time-order-dependent preprocessing
 * of FaintTrail 0.9.1 (jkobierczynski/FaintTrail), running on one NVIDIA B200
 * (sm_100a). Plain pointers and sizes only; host buffers are caller-owned and
 * never retained past the call. Images are row-major float32, a frame stack is
 * n consecutive w x h images. Every result is bit-identical to the reference CPU
 * backend on the same inputs.
 *
 * Status codes follow the reference C API (include/fainttrail/fainttrail.h:26-28):
 * FT_B200_OK, FT_B200_ERROR (message in ft_b200_last_error), FT_B200_CANCELLED
 * (a progress callback returned 0). A context is not thread-safe: one context
 * per host thread, like ft_context.
 */
#ifndef FT_B200_H
#define FT_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define FT_B200_OK 0
#define FT_B200_ERROR 1
#define FT_B200_CANCELLED 2
#define FT_B200_PENDING 3 /* ft_b200_server_poll: the request is not finished yet */

typedef struct ft_b200_ctx ft_b200_ctx;

/* Progress: fraction done in [0,1] and a stage name; return 0 to cancel.
 * Same shape as ft_progress_fn (fainttrail.h:72). */
typedef int (*ft_b200_progress_fn)(double fraction, const char* stage, void* user);

const char* ft_b200_version(void);

/* Open device `device` (-1: FAINTTRAIL_CUDA_DEVICE or 0, as the reference CUDA
 * backend resolves it, backend_cuda.cu:74-78). hbm_budget_bytes caps the device
 * memory the context allocates (0 = 90 % of the free memory). Blocks a call frees
 * stay with the context for the next call's allocations of the same sizes (at
 * most 48 GB, within the budget) until ft_b200_close, so the device memory in use
 * does not drop between calls; an allocation that fails returns them first. */
int ft_b200_open(int device, double hbm_budget_bytes, ft_b200_ctx** out);
void ft_b200_close(ft_b200_ctx* ctx);
/* Last error message of the context (ft_last_error, fainttrail.h:106); with a
 * NULL context, the last error on this thread of the entries that take no
 * context: ft_b200_open, ft_b200_server_open, ft_b200_stack_dev_noalloc,
 * ft_b200_set_tile_shape, ft_b200_null_threshold, ft_b200_pool_null_peaks,
 * ft_b200_write_candidates_csv and ft_b200_emulate_stack. */
const char* ft_b200_last_error(const ft_b200_ctx* ctx);
/* Device name, SM count and memory; replaces SearchBackend::description()
 * (backend.hpp:113). name_len bytes are written to name, NUL-terminated. */
int ft_b200_device_info(ft_b200_ctx* ctx, char* name, int name_len, int* sms, double* hbm_bytes);

/* One stacking pass: SearchBackend::run (backend.hpp:107-117; CPU reference
 * backend_cpu.cpp:77-204) with an explicit shift table (ShiftTable,
 * backend.hpp:56-69): motion j, frame i at dx[j * nframes + i]. frames: host,
 * nframes x height x width. Outputs max_snr and best_v (height x width, host),
 * exactly StackResult (backend.hpp:99-105). Malformed passes are refused as
 * validate_pass does (backend.cpp:89-108). progress may be NULL. */
int ft_b200_stack(ft_b200_ctx* ctx, const float* frames, int width, int height, int nframes, const int* dx,
                  const int* dy, int motions, int min_count, float* max_snr, int* best_v,
                  ft_b200_progress_fn progress, void* user);

/* The same with straight-line shifts round(v t) (pass_shift, backend.hpp:87-97):
 * t_h[nframes] in hours, velocities[2 * motions] as (vx, vy) pairs in px/hour. */
int ft_b200_stack_linear(ft_b200_ctx* ctx, const float* frames, int width, int height, int nframes,
                         const double* t_h, const double* velocities, int motions, int min_count, float* max_snr,
                         int* best_v, ft_b200_progress_fn progress, void* user);

/* Device-resident pass for callers that keep frames in HBM: d_frames is a device
 * pointer to nframes x height rows of `pitch` floats (pitch >= width, pitch * 4 a
 * multiple of 16, base 16-byte aligned); dx/dy are host tables as above;
 * d_max_snr / d_best_v are device outputs (height x width, dense). Runs on the
 * context's stream and returns when the pass is complete. */
int ft_b200_stack_dev(ft_b200_ctx* ctx, const float* d_frames, int width, int height, int pitch, int nframes,
                      const int* dx, const int* dy, int motions, int min_count, float* d_max_snr, int* d_best_v);

/* A stacking pass that allocates no device memory, for callers that cannot:
 * applications whose own arena or pool owns the GPU's memory and does not let a
 * library grow it, and latency-bound loops that must not wait on the allocator.
 * This entry point has no counterpart in FaintTrail; it is the device-resident
 * pass of ft_b200_stack_dev with the same arguments and results, needing no
 * context. The caller owns d_frames (nframes x height rows of `pitch` floats,
 * pitch >= width, pitch * 4 a multiple of 16, base 16-byte aligned) and the
 * outputs d_max_snr / d_best_v (height x width). dx/dy are host tables.
 * cuda_stream: a cudaStream_t of the current device (another device's stream is
 * refused), or NULL for the default stream. The call copies the pass's tables
 * from host memory, launches the pass, synchronises the stream and returns when
 * the pass is complete.
 * The pass's scratch -- its plan tables and launch descriptors -- lives in one
 * 32 MiB device array built into this library (every GPU that loads the library
 * holds it until the process exits); a pass whose tables need more (about 5
 * million motion x frame pairs) is refused with an error, nothing else is
 * limited. The first call on a device does a one-time set-up (it looks up that
 * array's device address on the device), so make the first call before any
 * stream capture begins. All calls share the array and it keeps the last call's
 * tables: calls that overlap on the GPU (other host threads, other streams) race
 * and must be serialised by the caller. Error text: ft_b200_last_error(NULL). */
int ft_b200_stack_dev_noalloc(const float* d_frames, int width, int height, int pitch, int nframes, const int* dx,
                              const int* dy, int motions, int min_count, float* d_max_snr, int* d_best_v,
                              void* cuda_stream);

/* One stacking pass computed on the host exactly as the device kernel computes
 * it, for checks of the pass planner on a machine without a GPU (the role of the
 * reference's emulate_cuda_pass, cuda_plan.cpp:74-117): the pass is planned for
 * kernel shape `shape` (1..7 as ft_b200_set_tile_shape; 0: the automatic choice)
 * with a B200's 227 KB of shared memory per block, and the plan -- tiles, motion
 * groups, frame windows zero-filled outside the frame, 16-bit window offsets,
 * coverage counts with the interior-tile shortcut, float adds in ascending frame
 * order, the maximum rule -- is walked on the CPU. Arguments and outputs as
 * ft_b200_stack (host buffers); slow (one CPU thread). No device is used; error
 * text in ft_b200_last_error(NULL). */
int ft_b200_emulate_stack(const float* frames, int width, int height, int nframes, const int* dx, const int* dy,
                          int motions, int min_count, int shape, float* max_snr, int* best_v);

/* The planner's view of a pass, for checks without a GPU (host only; no
 * counterpart in FaintTrail, whose CUDA plan has no motion groups): stats[0]
 * motion groups, [1] groups whose blocks share their column in every frame (the
 * kernel's row-descriptor path), [2] slots, [3] pad slots, [4] slots in those
 * groups, [5] the largest group's shared-memory bytes. shape as
 * ft_b200_emulate_stack. */
int ft_b200_plan_stats(int width, int height, int nframes, const int* dx, const int* dy, int motions, int shape,
                       long long* stats);

/* Test support for the stacking kernel's bounded waits (no counterpart in
 * FaintTrail): with extra_bytes > 0 every later stacking launch in the process
 * makes its staging barrier expect extra_bytes that no copy brings, so each
 * wait gives up after wait_cycles clock cycles, sets the device error flag and
 * the kernel returns; the pass then fails with "a device wait timed out" and the
 * context stays usable. extra_bytes 0 restores normal launches. */
int ft_b200_set_wait_test(int extra_bytes, long long wait_cycles);

/* Parameters of the preprocessing stage; the defaults are SearchParams'
 * (include/fainttrail/search.hpp:18-90): static_exclude -1 (= max(1, lround(n/8))),
 * clip 8, cosmic-ray level 5, mask scatter 2.5, weight scatter 1.5. fwhm_px is the
 * PSF FWHM in pixels and must be > 0 (the stage does not estimate it). */
typedef struct ft_b200_stage_params {
    double fwhm_px;
    int static_exclude;
    double clip_sigma;
    double cr_sigma;
    double mask_scatter;
    double weight_scatter;
} ft_b200_stage_params;

void ft_b200_stage_params_default(ft_b200_stage_params* p);

/* The time-order-dependent preprocessing: detail::build_stage (internal.hpp:55-58,
 * preprocess.cpp:286-486) on background-subtracted frames `sub` (host,
 * nframes x height x width, NaN = blank) observed at t_h[nframes] hours, with a
 * fixed PSF width (the form every null run uses, preprocess.cpp:488-521).
 * Outputs (host, any may be NULL): filtered (nframes x height x width, the
 * unit-variance matched-filtered frames), static_sky and mask (height x width),
 * sigma[nframes] (residual noise) and cr_pixels[nframes] (cosmic-ray hits).
 * At most 255 frames. */
int ft_b200_stage(ft_b200_ctx* ctx, const float* sub, int width, int height, int nframes, const double* t_h,
                  const ft_b200_stage_params* params, float* filtered, float* static_sky, float* mask, double* sigma,
                  int* cr_pixels);
/* The same for frames kept in HBM: d_sub is nframes x height rows of `pitch`
 * floats (pitch >= width) on the device, read only; d_filtered (the same
 * layout), d_static_sky and d_mask (height rows of `pitch` floats) are device
 * outputs, sigma and cr_pixels host arrays; any output may be NULL. Returns when
 * the outputs are complete. */
int ft_b200_stage_dev(ft_b200_ctx* ctx, const float* d_sub, int width, int height, int pitch, int nframes,
                      const double* t_h, const ft_b200_stage_params* params, float* d_filtered,
                      float* d_static_sky, float* d_mask, double* sigma, int* cr_pixels);

/* Parameters of a search: ft_params (fainttrail.h:32-54) plus the null-model
 * fields of SearchParams (search.hpp:58-68). Defaults: ft_b200_search_params_default,
 * equal to the reference's SearchParams defaults. `threads` is accepted and
 * ignored (the reference's CPU thread count). */
typedef struct ft_b200_search_params {
    double vmin_pxh, vmax_pxh, grid_tol_px, fwhm_px;
    double clip_sigma, cr_sigma, mask_scatter, weight_scatter, min_coverage;
    double threshold_snr, min_snr_floor, target_false_per_run, max_frame_fraction, half_tolerance;
    int static_exclude, null_runs, max_candidates, edge_px, threads;
    unsigned long long seed;
    int null_tested;      /* strongest null peaks per run screened for artefacts (3000) */
    int null_model_gauss; /* 1: "gauss" tail model (default), 0: "linear" */
    int passes_per_launch; /* 0 (default): every pass that fits the HBM budget in one
                              persistent launch; k > 0: at most k passes per launch,
                              the real pass alone first (1 = one pass per launch) */
    int shard_index, shard_count; /* null runs split over shard_count calls, one per GPU
                              (default 0, 1: no split). Call k runs null runs
                              [runs*k/count, runs*(k+1)/count) with the permutations
                              an unsplit search would give them. A shard's result
                              holds its pooled null peaks (method "shard",
                              no real pass): concatenate the shards' null peaks in
                              shard order, then ft_b200_null_threshold gives the
                              unsplit threshold; one call with it as
                              calibrated_threshold finishes the search. */
    double calibrated_threshold; /* > 0: the null-run threshold is given (no null runs
                              are run): the real pass, its peaks above min_snr_floor,
                              the selection at this threshold and the refined
                              candidates, as the unsplit search gives them */
    double calibrated_tail[4];   /* a, b, k, inv_s2 of that threshold's null-tail fit
                              (the candidates' false-alarm rates) */
    int align;            /* SearchParams::align (search.hpp:76-81, prepare_frames
                              preprocess.cpp:589-630): 0 "off" (default here): the
                              frames are taken as registered; 1 "check": the
                              registration check runs first (ft_b200_check_registration)
                              and frames that are not registered are an error with the
                              reference's message; 2 "auto": the same check, and frames
                              that are not registered are an error (the reference would
                              align them; this backend does not resample frames).
                              The check's outcome: ft_b200_result_registration. */
    const double* reg_dx; /* per-frame registration offsets (detector = registered +
                              offset), in the order the frames are passed, from the
                              FITS keywords REGDX / REGDY (Frame::reg_dx, types.hpp:61-65);
    */
    const double* reg_dy; /* with them the artefact screen of the null runs and the
                              candidates' flags include the detector test
                              (detector_flag, search.cpp:196-225). NULL (default): none. */
} ft_b200_search_params;

void ft_b200_search_params_default(ft_b200_search_params* p);

/* A detection-map peak (detail::Peak, internal.hpp:88-92): 0-based pixel,
 * coarse S/N, index of the trial motion. */
typedef struct ft_b200_peak {
    int x, y;
    float snr;
    int vidx;
} ft_b200_peak;

typedef struct ft_b200_result ft_b200_result;

/* The injection-recovery test, as completeness() (validate.cpp:62-165): the
 * threshold calibrated on the data (a full search), then per S/N level
 * per_level objects placed by the seeded xoshiro256** generator (at least
 * min_separation apart and from the objects the data holds), injected as
 * trailed Gaussians, searched with the threshold fixed and no null runs (all
 * levels' copies in one batch) and matched to the candidates within 2 px and
 * max(3, 2 dv) px/h. rows: nlevels entries. */
typedef struct ft_b200_completeness_row {
    double target_snr;
    int injected, recovered, detected; /* recovered: matched candidates that passed every test */
    double mean_snr, mean_dpos, mean_dv;
} ft_b200_completeness_row;

int ft_b200_completeness(ft_b200_ctx* ctx, const float* frames, int width, int height, int nframes, const double* mjd,
                         const double* exptime, const ft_b200_search_params* params, const double* snr_levels,
                         int nlevels, int per_level, double min_separation, unsigned long long seed,
                         ft_b200_completeness_row* rows, double* threshold_snr, char* method, int method_cap,
                         int* baseline_ok, double* snr50);

/* One null run's pooled S/N list from its raster-ordered peaks (host only):
 * order_peaks (std::sort by S/N, truncation at `keep`), the first `tested`
 * screened with the given artefact flags (artefact[q] for raster peak q), then
 * pool_null_peaks (search.cpp:766-781, 690-693). mode 0: the reference's full
 * sort; mode 1: the search's path (the screened set by nth_element, the full
 * sort only for a tie at the screening boundary). Writes up to cap values into
 * pooled and returns their count. */
int ft_b200_pool_null_peaks(const ft_b200_peak* raster, int count, const unsigned char* artefact, int keep,
                            int tested, int mode, float* pooled, int cap);

/* The null-tail threshold from pooled null-peak S/N values (set_threshold,
 * search.cpp:573-612; fit_null_tail_gauss :471-510, gauss_tail_level :517-527):
 * `pooled` is every run's surviving null peaks, run after run, `runs` the number
 * of null runs, `motions` the trial motions of the grid. Host only (no device
 * work, no context): the reduction step of a search whose null runs were split
 * over GPUs. method receives "null-fit gauss", "null-fit linear", "floor", ... */
int ft_b200_null_threshold(const double* pooled, long long count, int runs, double fwhm_px, int width, int height,
                           int motions, const ft_b200_search_params* params, double* threshold, char* method,
                           int method_cap, double* a, double* b, double* k, double* inv_s2);

/* A whole search from raw registered frames, as ft_search does (c_api.cpp:172-204:
 * frames stable-sorted by mid-exposure time, prepare, then search): background
 * and blank-border growth, preprocessing, the real stacking pass and its peaks,
 * params->null_runs time-shuffled null runs (preprocessing rebuilt, stacked,
 * peaks screened for artefacts), the null-tail fit and threshold, the peaks
 * selected for refinement and their refined candidates (search.cpp:716-804;
 * ft_b200_result_candidates). Sky coordinates and photometric calibration are
 * left to the caller. frames: host, nframes x height x width; mjd/exptime per frame.
 * On success *out receives a result to release with ft_b200_result_free. */
int ft_b200_search(ft_b200_ctx* ctx, const float* frames, int width, int height, int nframes, const double* mjd,
                   const double* exptime, const ft_b200_search_params* params, ft_b200_progress_fn progress,
                   void* user, ft_b200_result** out);

/* The tiled search (search_tiled, tiled.cpp:272-647; FrameSource tiled.hpp:42-54)
 * for sequences larger than HBM: the frames (host, as ft_b200_search) stay in
 * host memory and are uploaded in full-width bands of band_rows core rows (0:
 * 1024) grown by the reference's halos -- the longest trial shift for the
 * stacking, the filter and mask reach, the refinement's reach. The background,
 * residual noise and filter normalisation of every frame are measured on the
 * whole frame from the untiled search's sample positions, the bands' maps are
 * assembled before peaks are found, and the null runs' artefact screen and the
 * refinement run on bands in the whole image's coordinates: the result equals
 * ft_b200_search's bit for bit (maps, null peaks, threshold, candidates). The
 * registration check (align) is not run here; cosmic-ray counts are not kept. */
int ft_b200_search_tiled(ft_b200_ctx* ctx, const float* frames, int width, int height, int nframes, const double* mjd,
                         const double* exptime, const ft_b200_search_params* params, int band_rows,
                         ft_b200_progress_fn progress, void* user, ft_b200_result** out);
/* The same over frames already in device memory: d_frames holds nframes x height
 * rows of `pitch` floats (pitch >= width), is read only, and is copied in time
 * order. Synchronous; no progress callback. */
int ft_b200_search_dev(ft_b200_ctx* ctx, const float* d_frames, int width, int height, int pitch, int nframes,
                       const double* mjd, const double* exptime, const ft_b200_search_params* params,
                       ft_b200_result** out);
void ft_b200_result_free(ft_b200_result* r);
/* The refined candidates (refine() and finish_candidates(), search.cpp:245-400,
 * 620-676): 17 doubles per candidate into rows[17 * k ..] -- x, y, vx, vy,
 * pos_err, vel_err, snr, snr_coarse, snr_half1, snr_half2, max_frame_fraction,
 * false_alarms_per_run, flux, mag_inst, ok (0/1), id, inv_dist -- and the
 * comma-separated flags into flags[64 * k ..]; up to cap candidates; returns
 * the count. Sky coordinates are not computed (no WCS). */
int ft_b200_result_candidates(const ft_b200_result* r, double* rows, char* flags, int cap);

/* An object to inject into every frame of a copy: Injection (validate.hpp:18-23),
 * position at the reference epoch (0-based px), motion (px/hour), flux per frame. */
typedef struct ft_b200_injection {
    double x_ref, y_ref, vx_pxh, vy_pxh, flux;
} ft_b200_injection;

/* The search of ft_b200_search plus injection-recovery copies, all in one batch
 * (completeness's searches, validate.cpp:62-126): copy k holds the raw frames
 * with objects_per_copy[k] objects injected (ft_b200_injection, consecutive for
 * all copies; the trailed Gaussians of inject(), validate.cpp:17-29, rendered
 * with the reference's arithmetic), prepared again and searched with the
 * threshold the null runs calibrated held fixed, no null runs, and the same PSF
 * width. The real pass, the null runs and the copies are stacked together in
 * persistent launches. *base receives the search's result; copy_results[k] (an
 * array of `copies` pointers) each copy's result (peaks above the threshold,
 * selected peaks, maps). Release every result with ft_b200_result_free. */
int ft_b200_search_batch(ft_b200_ctx* ctx, const float* frames, int width, int height, int nframes,
                         const double* mjd, const double* exptime, const ft_b200_search_params* params, int copies,
                         const int* objects_per_copy, const ft_b200_injection* objects, ft_b200_progress_fn progress,
                         void* user, ft_b200_result** base, ft_b200_result** copy_results);
/* The same over frames already in device memory (nframes x height rows of
 * `pitch` floats, read only), as ft_b200_search_dev. Synchronous. */
int ft_b200_search_batch_dev(ft_b200_ctx* ctx, const float* d_frames, int width, int height, int pitch, int nframes,
                             const double* mjd, const double* exptime, const ft_b200_search_params* params,
                             int copies, const int* objects_per_copy, const ft_b200_injection* objects,
                             ft_b200_result** base, ft_b200_result** copy_results);
/* threshold_snr and the tail model (SearchResult, search.hpp:163-172); method
 * receives "fixed", "null-fit gauss", "null-fit linear", "null-quantile" or
 * "gaussian". Any pointer may be NULL. */
double ft_b200_result_threshold(const ft_b200_result* r, char* method, int method_len, double* null_a,
                                double* null_b, double* null_k, double* null_inv_s2);
/* fwhm_px, dv_pxh, t_ref_mjd and the number of trial motions of the search. */
int ft_b200_result_info(const ft_b200_result* r, double* fwhm_px, double* dv_pxh, double* t_ref_mjd,
                        int* n_velocities);
/* which = 0: all real-run peaks above the floor, S/N descending (find_peaks);
 * which = 1: the peaks selected for refinement (select_peaks). Returns the
 * count; writes at most cap. */
int ft_b200_result_peaks(const ft_b200_result* r, int which, ft_b200_peak* out, int cap);
/* The pooled null-peak S/N values (SearchResult::null_peaks). Returns the count. */
int ft_b200_result_null_peaks(const ft_b200_result* r, double* out, int cap);
/* One candidate as ft_get_candidate reports it (ft_candidate, fainttrail.h:55-68;
 * c_api.cpp:218-246), field for field: FITS 1-based x and y, ra_deg, dec_deg,
 * rate_arcsec_min and pa_deg 0 (no WCS). */
typedef struct ft_b200_candidate {
    int id;
    int ok;
    double x, y;
    double vx_pxh, vy_pxh;
    double pos_err_px, vel_err_pxh;
    double snr, snr_coarse, snr_half1, snr_half2;
    double max_frame_fraction;
    double false_alarms_per_run;
    double flux, mag_inst;
    double ra_deg, dec_deg;
    double rate_arcsec_min, pa_deg;
    char flags[64];
} ft_b200_candidate;
int ft_b200_result_candidate(const ft_b200_result* r, int index, ft_b200_candidate* out);
/* Predicted position of candidate `index` in frame `frame` (0-based, in time
 * order), as ft_get_track_point (fainttrail.h:102-104, c_api.cpp:248-261): the
 * frame's mid-exposure MJD and the FITS 1-based position on the straight track;
 * ra_deg and dec_deg 0 (no WCS). Any output may be NULL. */
int ft_b200_result_track_point(const ft_b200_result* r, int index, int frame, double* mjd, double* x, double* y,
                               double* ra_deg, double* dec_deg);
/* The candidate file of the search (write_candidates_csv, io.cpp:82-115), byte
 * for byte as the reference writes it for frames without a WCS, photometric
 * calibration or near-Earth distances: two comment lines (reference epoch,
 * threshold, motion grid, PSF width), the column names, and one line per
 * candidate with ra_deg, dec_deg, rate_arcsec_min and pa_deg 0 and empty mag,
 * mag_err and mag_band. ft_b200_write_candidates_csv writes it to path (error
 * text in ft_b200_last_error(NULL)); ft_b200_result_candidates_csv copies it to
 * buf (at most cap - 1 bytes and a NUL) and returns its length, or -1. */
int ft_b200_write_candidates_csv(const ft_b200_result* r, const char* path);
long long ft_b200_result_candidates_csv(const ft_b200_result* r, char* buf, long long cap);
/* The real run's detection map: max_snr and best_v, height x width each. */
int ft_b200_result_maps(const ft_b200_result* r, float* max_snr, int* best_v);
/* The trial motion vidx of the grid (velocity_grid, search.cpp:39-58), px/hour. */
int ft_b200_result_velocity(const ft_b200_result* r, int vidx, double* vx_pxh, double* vy_pxh);

/* The registration check of a frame sequence (DriftCheck, registration.hpp:22-30;
 * check_registration, registration.cpp:260-312): stars (bright, extended local
 * maxima) are found in the first, middle and last frame by time, the last and the
 * middle frame's are matched to the first's by an offset vote and a similarity
 * fit, and the sequence is registered when neither moves any point of the frame
 * by more than 1.5 px. Fewer than 3 frames, or too few stars to match: not
 * measured, and registered. */
typedef struct ft_b200_drift_check {
    int measured;          /* enough stars matched to tell */
    int registered;        /* 1 when not measured */
    int stars;             /* stars used in the first frame (at most 60) */
    int matched;           /* stars matched between the first and the last frame */
    double dx, dy;         /* displacement of the field centre, first -> last frame, px */
    double mid_dx, mid_dy; /* the same, first -> middle frame */
    double rate_pxh;       /* |(dx, dy)| / time between the first and the last frame */
    char message[1024];    /* why the frames are not registered ("" when they are) */
} ft_b200_drift_check;

/* The check on host frames (nframes x height x width floats, NaN = blank)
 * observed at t_h[nframes] hours (any order; the reference passes
 * (mjd_mid - mjd_mid of the first frame) * 24). Only the three frames the check
 * uses are copied to the device. */
int ft_b200_check_registration(ft_b200_ctx* ctx, const float* frames, int width, int height, int nframes,
                               const double* t_h, ft_b200_drift_check* out);
/* The same on device frames (frame i at d_frames + i * pitch * height, pitch >= width). */
int ft_b200_check_registration_dev(ft_b200_ctx* ctx, const float* d_frames, int width, int height, int pitch,
                                   int nframes, const double* t_h, ft_b200_drift_check* out);
/* The registration check a search ran (align 1 or 2); not measured and
 * registered when it ran none. */
int ft_b200_result_registration(const ft_b200_result* r, ft_b200_drift_check* out);

/* Stack kernel tile shape for every later pass in this process: 0 = automatic
 * (the default: the autotuned choice where one is cached for the pass's frame
 * count, else the first shape whose windows fit), 1 = 32 x 16 output tiles,
 * 2 = 64 x 8 tiles with paired columns, 3 = 32 x 8, 4 = 32 x 4, 5 and 6 = 32 x 16
 * with one shared maximum per tile (16 and 14 warps), 7 = 32 x 12, 8 = 32 x 20
 * with the shared maximum (16 warps). A fixed shape
 * whose frame windows do not fit shared memory falls back to automatic. Results
 * do not depend on the shape. No counterpart in the reference (its CUDA kernel
 * has one shape, backend_cuda.cu:55-72). */
int ft_b200_set_tile_shape(int shape);
int ft_b200_tile_shape(void);
/* The autotuner's choices so far: for a pass of at least 5e11 adds whose
 * (frames, motions, width, height) it has not seen, automatic mode plans every
 * shape that fits, times each on a band of tile rows in the middle of the image
 * and keeps the fastest per output pixel. Fills keys[4 * k .. 4 * k + 3] (frames,
 * motions, width, height) and shapes[k] for up to cap entries; returns the count.
 * ft_b200_clear_tuned_shapes forgets them. */
int ft_b200_tuned_shapes(int* keys, int* shapes, int cap);
void ft_b200_clear_tuned_shapes(void);

/* The serving loop. A server owns worker threads, each with its own device
 * context and stream; requests (frames of any count and size, any motion range)
 * are copied into HBM on submission and stay resident there until they are
 * prepared (in host memory instead while the resident frames would take more
 * than half the HBM budget). Workers run steps: at every step a worker admits
 * queued requests in arrival order as the HBM budget allows and prepares them,
 * then stacks up to max_batch passes (real passes and null runs with their
 * rebuilt preprocessing) taken in turn from all its admitted requests in shared
 * persistent launches, and publishes the requests whose passes are all done. A
 * request that arrives while others are on the GPU is admitted at the next step
 * and its passes share launches with theirs. Each result equals ft_b200_search
 * on the same request. This has no counterpart in the reference, which runs one
 * search at a time (search.cpp:716). max_batch caps the passes per step and the
 * requests a worker holds. */
typedef struct ft_b200_server ft_b200_server;

/* workers: steps in flight at once (each on its own stream; <= 0: 2), so one
 * step's host work overlaps another's kernels. The workers share the HBM budget:
 * requests are admitted while their estimated memory (prepared frames plus a
 * step's passes) fits what the admitted ones and the resident frames leave, and
 * one that needs the whole budget runs alone. */
int ft_b200_server_open(int device, double hbm_budget_bytes, int max_batch, int workers, ft_b200_server** out);
/* Finishes the queued requests, then stops the worker. */
void ft_b200_server_close(ft_b200_server* s);
int ft_b200_server_submit(ft_b200_server* s, const float* frames, int width, int height, int nframes,
                          const double* mjd, const double* exptime, const ft_b200_search_params* params,
                          long long* request_id);
/* FT_B200_OK with *out set when the request is done; FT_B200_PENDING if not done
 * within wait_ms (0: do not wait, < 0: wait until done); FT_B200_ERROR if it
 * failed or the id is unknown (message: ft_b200_server_error). A finished
 * request is handed out once. */
int ft_b200_server_poll(ft_b200_server* s, long long request_id, int wait_ms, ft_b200_result** out);
const char* ft_b200_server_error(const ft_b200_server* s);
/* Hold (1) or resume (0) admission; held requests queue up and start together. */
int ft_b200_server_pause(ft_b200_server* s, int paused);
/* Completed requests, their p50 / p99 latency (submit to done, seconds),
 * throughput (completed / time from first submit to last completion), steps
 * (rounds), mean requests per step and kernels launched. */
int ft_b200_server_stats(ft_b200_server* s, long long* completed, double* p50_s, double* p99_s,
                         double* searches_per_s, long long* rounds, double* mean_batch, long long* launches);

/* Kernels launched by the last call on the context (its stacking passes, stage,
 * peak and screening kernels). pixel_adds is reserved (left unchanged). */
int ft_b200_stats(const ft_b200_ctx* ctx, long long* kernel_launches, double* pixel_adds);

/* Stage timings of the last call on the context, measured with CUDA events on the
 * context's stream (the reference's StackResult::timings, backend.hpp:99-105, and
 * Prepared::timings, search.hpp:118): names as one ';'-separated string in
 * `names` (names_len bytes), seconds[k] for each; returns the number of stages. */
int ft_b200_timings(const ft_b200_ctx* ctx, char* names, int names_len, double* seconds, int cap);

#ifdef __cplusplus
}
#endif

#endif /* FT_B200_H */
