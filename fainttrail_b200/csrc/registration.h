// The registration check of a frame sequence (FaintTrail check_registration,
// registration.cpp:260-312): stars found on the device in the first, middle and
// last frame by time, then matched and fitted on the host (registration_host.h).
#pragma once

#include "engine.h"
#include "registration_host.h"

namespace ftb {

// check_registration on n device frames d_frames (frame i at d_frames + i *
// plane, rows `pitch` floats apart) observed at t_h[n] hours. Fewer than 3
// frames: not measured.
DriftCheck check_registration_device(Context& c, const float* d_frames, size_t plane, int pitch, int w, int h, int n,
                                     const double* t_h);

// The same on the three frames it uses (first, middle, last by time; device,
// rows `pitch` floats apart) and the time from the first to the last in hours.
DriftCheck check_registration_three(Context& c, const float* const frames[3], int pitch, int w, int h, double dt_h);

}  // namespace ftb
