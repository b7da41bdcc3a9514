#include "host_util.h"

#include <cmath>

namespace pt {

namespace {
struct F3 {
    float x, y, z;
};
inline F3 sub(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline F3 crs(F3 a, F3 b) {
    return {a.y * b.z - a.z * b.y, -(a.x * b.z - a.z * b.x), a.x * b.y - a.y * b.x};
}
inline F3 nrm(F3 v) {
    const float l = std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z);
    return {v.x / l, v.y / l, v.z / l};
}

// One row (or the marginal) of the CDF: FP64 prefix sums over `n` values, written as FP32.
void cdf_row(const double* v, int n, float* cdf, double& mass_out) {
    double mass = 0.0;
    for (int i = 0; i < n; i++) mass += v[i];
    mass_out = mass;
    if (!(mass > 0.0)) {
        for (int i = 0; i < n; i++) cdf[i] = 0.f;
        return;
    }
    int last = -1;
    double run = 0.0;
    for (int i = 0; i < n; i++) {
        if (v[i] > 0.0) last = i;
        run += v[i];
        cdf[i] = (float)(run / mass);
    }
    for (int i = last; i < n; i++) cdf[i] = 1.0f;
}
}  // namespace

bool make_camera(const CameraSpec& spec, int res_x, int res_y, CameraParams& out, std::string& err) {
    if (res_x <= 0 || res_y <= 0) {
        err = "resolution must be positive";
        return false;
    }
    const F3 src{spec.origin[0], spec.origin[1], spec.origin[2]};
    const F3 tgt{spec.target[0], spec.target[1], spec.target[2]};
    const F3 up{spec.up[0], spec.up[1], spec.up[2]};
    const F3 dir = nrm(sub(src, tgt));
    if (dir.x == up.x && dir.y == up.y && dir.z == up.z) {
        err = "look direction cannot equal the up vector";
        return false;
    }
    const F3 xa = nrm(crs(nrm(up), dir));
    const F3 ya = nrm(crs(dir, xa));
    if (!std::isfinite(xa.x) || !std::isfinite(ya.x) || !std::isfinite(dir.x)) {
        err = "degenerate camera frame";
        return false;
    }
    const float sign = spec.flip ? -1.f : 1.f;
    out = CameraParams();
    const float m[3][4] = {{sign * xa.x, ya.x, dir.x, src.x},
                           {sign * xa.y, ya.y, dir.y, src.y},
                           {sign * xa.z, ya.z, dir.z, src.z}};
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 4; c++) out.m[r][c] = m[r][c];
    out.top = std::tan(spec.vfov / 2.f);
    out.height = out.top * 2.f;
    const float aspect = 1.f * res_x / res_y;
    out.width = out.height * aspect;
    out.right = out.width / 2.f;
    out.res_x = res_x;
    out.res_y = res_y;
    out.vfov = spec.vfov;
    out.flip = spec.flip ? 1 : 0;
    for (int k = 0; k < 3; k++) {
        out.origin[k] = spec.origin[k];
        out.target[k] = spec.target[k];
        out.up[k] = spec.up[k];
    }
    return true;
}

void build_env_cdf(const float* rgba, int w, int h, EnvCdf& out) {
    out.marg.assign(h, 0.f);
    out.cond.assign((size_t)w * h, 0.f);
    out.row_mass.assign(h, 0.f);
    std::vector<double> row(w), masses(h);
    for (int y = 0; y < h; y++) {
        for (int x = 0; x < w; x++) {
            const float* t = &rgba[((size_t)y * w + x) * 4];
            row[x] = (double)t[0] + (double)t[1] + (double)t[2];
        }
        double m;
        cdf_row(row.data(), w, &out.cond[(size_t)y * w], m);
        masses[y] = m;
        out.row_mass[y] = (float)m;
    }
    double total;
    cdf_row(masses.data(), h, out.marg.data(), total);
    out.total = (float)total;
}

}  // namespace pt
