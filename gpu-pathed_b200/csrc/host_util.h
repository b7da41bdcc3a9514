// Host-side helpers: camera matrix (lookAt) and the environment-map importance CDF.
#pragma once

#include <string>
#include <vector>

#include "host_scene.h"
#include "pt_types.h"

namespace pt {

// Camera parameters for generateRay (include/core/camera.h:40-61) from a CameraSpec, using
// lookAt's construction (src/transform.cu:7-33) in single precision. Returns false when the
// look direction equals the up vector (the reference exits the process there, :15-18).
bool make_camera(const CameraSpec& spec, int res_x, int res_y, CameraParams& out, std::string& err);

// Marginal/conditional CDF of an equirect map, luminance = R + G + B
// (src/lights/environment_light.cu:44-47). Prefix sums and normalisation in FP64; stored as
// FP32 with the reference's tail rule: every entry from the last non-zero one onwards is
// exactly 1.0 (src/math/distribution.cu:19-55). Rows without mass keep row_mass = 0 and an
// all-zero conditional CDF; they have zero marginal probability and are never sampled.
struct EnvCdf {
    std::vector<float> marg;      // H
    std::vector<float> cond;      // H * W
    std::vector<float> row_mass;  // H
    float total = 0.f;
};
void build_env_cdf(const float* rgba, int w, int h, EnvCdf& out);

}  // namespace pt
