// Internal declarations shared by the host-side translation units of libglc.
#pragma once

#include "../../include/glc.h"

namespace glc {

// Records a thread-local error message and returns the status (for `return set_error(...)`).
glc_status set_error(glc_status status, const char* message);

glc_status pack_scene(const glc_scene_input& in, glc_scene& out);
double prograde_isco(double a, double q);
void flop_model(double out[4]);

}  // namespace glc
