// A refined candidate and the candidate list file of a search. Plain C++ with
// no CUDA dependency, so that host-only tests build the file writer too.
#pragma once

#include <string>
#include <vector>

namespace ftb {

// A refined candidate (Candidate, search.hpp:131-154) without sky coordinates
// or calibrated magnitudes (this backend has no WCS or photometry).
struct Candidate {
    int id = 0;
    double x = 0, y = 0, vx_pxh = 0, vy_pxh = 0, pos_err_px = 0, vel_err_pxh = 0;
    double snr = 0, snr_coarse = 0, snr_half1 = 0, snr_half2 = 0, max_frame_fraction = 0;
    double false_alarms_per_run = 0, flux = 0, mag_inst = 0, inv_dist_au = 0;
    bool ok = false;
    std::string flags;
};

// Where a candidate is predicted in a frame observed t_h hours after the
// reference epoch, as ft_get_track_point reports it (c_api.cpp:248-261,
// track_points search.cpp:893-905, track_pos internal.hpp:107-116): the
// frame's MJD and the FITS 1-based position of the straight track.
struct TrackPoint {
    double mjd, x, y;
};

inline TrackPoint track_point(double t_ref_mjd, double t_h, const Candidate& c) {
    TrackPoint p;
    p.mjd = t_ref_mjd + t_h / 24.0;
    const double x = c.x + c.vx_pxh * t_h, y = c.y + c.vy_pxh * t_h;
    p.x = x + 1.0;
    p.y = y + 1.0;
    return p;
}

// The search-level values the candidate file's header line carries.
struct CandidateListInfo {
    double t_ref_mjd = 0.0, threshold_snr = 0.0, dv_pxh = 0.0, fwhm_px = 0.0;
    std::string method;
    long long n_velocities = 0;
};

// The candidate file as write_candidates_csv (io.cpp:82-115) writes it for a
// search without a WCS, photometric calibration or near-Earth distances: two
// comment lines, the column names, one line per candidate with its sky
// coordinates, rate and position angle 0 and empty magnitude columns.
std::string candidates_csv(const CandidateListInfo& info, const std::vector<Candidate>& cands);

// ISO 8601 UTC of an MJD with `decimals` decimals of seconds (iso_from_mjd,
// fits.cpp:474-504).
std::string iso_utc_from_mjd(double mjd, int decimals);

}  // namespace ftb
