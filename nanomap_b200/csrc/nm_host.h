// nm_host.h -- host-side math shared by the C ABI translation units.
#pragma once

#include "nanomap_b200.h"

namespace nm {

// world-from-sensor rotation (row-major) = rot(q / |q|) * F, F column-major; double, then
// rounded once to float.
void pose_rotation(const nm_pose& pose, const float F[9], float R[9]);
// index-space eye (position times the inverse voxel size) and max_time = max_range / res,
// both under the map's rounding policy.
void frame_constants(const nm_pose& pose, float res, float max_range, int rounding, double eye[3],
                     float* max_time);
// frustum pixel model: hw, hh, 2hw, 2hh, 1/W, 1/H
void frustum_params(int W, int H, float hfov_deg, float vfov_deg, float out[6]);
// laser grid sines and cosines (double, rounded to float)
void laser_tables(int W, int H, float hfov_deg, float vfov_deg, float* sinu, float* cosu,
                  float* sinv, float* cosv);
float logit(float p);

}  // namespace nm
