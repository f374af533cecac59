// Test infrastructure only: the candidate file writer
// (fainttrail_b200/csrc/candidate_csv.cpp) built for the host, fed with the
// reference's result fields, so that the CPU tests compare its text with the
// reference's write_candidates_csv (io.cpp:82-115) on a machine without a GPU.
#include <cstring>
#include <vector>

#include "candidate.h"

// info = t_ref_mjd, threshold_snr, dv_pxh, fwhm_px, n_velocities; rows: n x 17
// (x, y, vx, vy, pos_err, vel_err, snr, snr_coarse, snr_half1, snr_half2,
// max_frame_fraction, false_alarms_per_run, flux, mag_inst, ok, id, inv_dist);
// flags: n x 64 bytes. Writes the text into out (cap bytes, NUL-terminated) and
// returns its length.
extern "C" long long ftb_host_candidates_csv(const double* info, const char* method, const double* rows,
                                             const char* flags, int n, char* out, long long cap) {
    ftb::CandidateListInfo in;
    in.t_ref_mjd = info[0];
    in.threshold_snr = info[1];
    in.dv_pxh = info[2];
    in.fwhm_px = info[3];
    in.n_velocities = static_cast<long long>(info[4]);
    in.method = method;
    std::vector<ftb::Candidate> cands(static_cast<size_t>(n));
    for (int k = 0; k < n; ++k) {
        const double* r = rows + 17 * k;
        ftb::Candidate& c = cands[static_cast<size_t>(k)];
        c.x = r[0];
        c.y = r[1];
        c.vx_pxh = r[2];
        c.vy_pxh = r[3];
        c.pos_err_px = r[4];
        c.vel_err_pxh = r[5];
        c.snr = r[6];
        c.snr_coarse = r[7];
        c.snr_half1 = r[8];
        c.snr_half2 = r[9];
        c.max_frame_fraction = r[10];
        c.false_alarms_per_run = r[11];
        c.flux = r[12];
        c.mag_inst = r[13];
        c.ok = r[14] != 0.0;
        c.id = static_cast<int>(r[15]);
        c.inv_dist_au = r[16];
        c.flags = std::string(flags + 64 * k, strnlen(flags + 64 * k, 64));
    }
    const std::string text = ftb::candidates_csv(in, cands);
    if (out && cap > 0) {
        const size_t m = text.size() < static_cast<size_t>(cap - 1) ? text.size() : static_cast<size_t>(cap - 1);
        std::memcpy(out, text.data(), m);
        out[m] = 0;
    }
    return static_cast<long long>(text.size());
}

// track_point of every candidate (rows as above) in every frame (t_h[n]):
// out[(k * n + i) * 5 ..] = mjd, x, y (FITS 1-based), ra 0, dec 0.
extern "C" void ftb_host_track_points(double t_ref_mjd, const double* t_h, int n, const double* rows, int nc,
                                      double* out) {
    for (int k = 0; k < nc; ++k) {
        ftb::Candidate c;
        c.x = rows[17 * k];
        c.y = rows[17 * k + 1];
        c.vx_pxh = rows[17 * k + 2];
        c.vy_pxh = rows[17 * k + 3];
        for (int i = 0; i < n; ++i) {
            const ftb::TrackPoint p = ftb::track_point(t_ref_mjd, t_h[i], c);
            double* o = out + (static_cast<size_t>(k) * n + i) * 5;
            o[0] = p.mjd;
            o[1] = p.x;
            o[2] = p.y;
            o[3] = 0.0;
            o[4] = 0.0;
        }
    }
}

// iso_utc_from_mjd for the date checks.
extern "C" void ftb_host_iso_utc(double mjd, int decimals, char* out, int cap) {
    const std::string s = ftb::iso_utc_from_mjd(mjd, decimals);
    std::strncpy(out, s.c_str(), static_cast<size_t>(cap) - 1);
    out[cap - 1] = 0;
}
