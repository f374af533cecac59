// The candidate list file of a search (FaintTrail write_candidates_csv,
// io.cpp:82-115), byte for byte as the reference writes it for a search without
// a WCS, photometric calibration or near-Earth distances. The reference prints
// through an ostream in fixed notation with per-column precisions; the same
// digits come from printf's %.Nf / %.Ne, which that ostream formatting uses.
#include <cmath>
#include <cstdio>

#include "candidate.h"

namespace ftb {

namespace {

void put_fixed(std::string& s, double v, int digits) {
    char buf[400];  // %.Nf of any double fits
    std::snprintf(buf, sizeof buf, "%.*f", digits, v);
    s += buf;
}

void put_sci(std::string& s, double v, int digits) {
    char buf[64];
    std::snprintf(buf, sizeof buf, "%.*e", digits, v);
    s += buf;
}

}  // namespace

std::string iso_utc_from_mjd(double mjd, int decimals) {
    // seconds of the day rounded to the printed decimals, carried into the next
    // day at 86400 (fits.cpp:475-482)
    double days = std::floor(mjd);
    double sec = (mjd - days) * 86400.0;
    const double scale = std::pow(10.0, decimals);
    sec = std::round(sec * scale) / scale;
    if (sec >= 86400.0) {
        sec -= 86400.0;
        days += 1.0;
    }
    // the civil date of a day count: H. Hinnant's days-to-civil algorithm
    // (eras of 400 years from 0000-03-01), on days since 1970-01-01
    // (MJD 40587)
    const long long z = static_cast<long long>(days) - 40587 + 719468;
    const long long era = (z >= 0 ? z : z - 146096) / 146097;
    const unsigned doe = static_cast<unsigned>(z - era * 146097);
    const unsigned yoe = (doe - doe / 1460 + doe / 36524 - doe / 146096) / 365;
    const unsigned doy = doe - (365 * yoe + yoe / 4 - yoe / 100);
    const unsigned mp = (5 * doy + 2) / 153;
    const unsigned day = doy - (153 * mp + 2) / 5 + 1;
    const unsigned month = mp < 10 ? mp + 3 : mp - 9;
    const long long year = static_cast<long long>(yoe) + era * 400 + (month <= 2 ? 1 : 0);
    const int hh = static_cast<int>(sec / 3600.0);
    const int mm = static_cast<int>((sec - hh * 3600.0) / 60.0);
    const double ss = sec - hh * 3600.0 - mm * 60.0;
    char buf[96];
    if (decimals > 0)
        std::snprintf(buf, sizeof buf, "%04lld-%02u-%02uT%02d:%02d:%0*.*f", year, month, day, hh, mm, decimals + 3,
                      decimals, ss);
    else
        std::snprintf(buf, sizeof buf, "%04lld-%02u-%02uT%02d:%02d:%02d", year, month, day, hh, mm,
                      static_cast<int>(std::lround(ss)));
    return buf;
}

std::string candidates_csv(const CandidateListInfo& info, const std::vector<Candidate>& cands) {
    std::string s = "# fainttrail candidates; pixel coordinates are FITS 1-based at the reference epoch\n";
    s += "# t_ref_mjd=";
    put_fixed(s, info.t_ref_mjd, 8);
    s += " t_ref_utc=" + iso_utc_from_mjd(info.t_ref_mjd, 2) + " threshold_snr=";
    put_fixed(s, info.threshold_snr, 3);
    s += " method=" + info.method + " velocities=" + std::to_string(info.n_velocities) + " dv_pxh=";
    put_fixed(s, info.dv_pxh, 3);
    s += " fwhm_px=";
    put_fixed(s, info.fwhm_px, 3);
    s += "\n";
    s += "id,ok,flags,x,y,pos_err_px,vx_pxh,vy_pxh,vel_err_pxh,snr,snr_coarse,snr_half1,snr_half2,max_frame_fraction,"
         "false_alarms_per_run,flux,mag_inst,ra_deg,dec_deg,rate_arcsec_min,pa_deg,mag,mag_err,mag_band\n";
    for (const Candidate& c : cands) {
        s += std::to_string(c.id) + (c.ok ? ",1,\"" : ",0,\"") + c.flags + "\",";
        // position (FITS 1-based), motion and their errors: 3 decimals
        for (const double v : {c.x + 1.0, c.y + 1.0, c.pos_err_px, c.vx_pxh, c.vy_pxh, c.vel_err_pxh}) {
            put_fixed(s, v, 3);
            s += ',';
        }
        // S/N values: 2 decimals
        for (const double v : {c.snr, c.snr_coarse, c.snr_half1, c.snr_half2}) {
            put_fixed(s, v, 2);
            s += ',';
        }
        put_fixed(s, c.max_frame_fraction, 3);
        s += ',';
        put_sci(s, c.false_alarms_per_run, 2);
        s += ',';
        put_fixed(s, c.flux, 2);
        s += ',';
        put_fixed(s, c.mag_inst, 3);
        s += ',';
        // no WCS: sky position, rate and position angle stay 0 (search.cpp:438-439)
        put_fixed(s, 0.0, 7);
        s += ',';
        put_fixed(s, 0.0, 7);
        s += ',';
        put_fixed(s, 0.0, 4);
        s += ',';
        put_fixed(s, 0.0, 2);
        // no photometric calibration: empty mag, mag_err and mag_band
        s += ",,,\n";
    }
    return s;
}

}  // namespace ftb
