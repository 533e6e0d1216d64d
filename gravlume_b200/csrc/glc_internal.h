// Internal declarations shared by the host-side translation units of libglc.
#pragma once

#include "../../include/glc.h"

namespace glc {

// Records a thread-local error message and returns the status (for `return set_error(...)`).
glc_status set_error(glc_status status, const char* message);

glc_status pack_scene(const glc_scene_input& in, glc_scene& out);

// The policy checks of glc_set_policy, and the per-camera checks and padded ray count of every
// trace entry point (its tile region for image cameras).
glc_status check_policy(const glc_policy& p);
glc_status camera_ray_count(const glc_camera& c, const glc_scene* scenes, int32_t n_scenes, const glc_policy& pol,
                            unsigned long long* n);
double prograde_isco(double a, double q);
void flop_model(double out[4]);

}  // namespace glc
