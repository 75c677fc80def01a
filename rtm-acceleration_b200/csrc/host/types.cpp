// types.cpp -- value-type helpers and the shared numerics of the C++ host API.
#include <algorithm>
#include <cmath>
#include <stdexcept>

#include "rtm_b200_engine.hpp"

namespace rtm_b200 {

float VelocityModel::vmin() const { return v.empty() ? 0.0f : *std::min_element(v.begin(), v.end()); }
float VelocityModel::vmax() const { return v.empty() ? 0.0f : *std::max_element(v.begin(), v.end()); }

std::vector<float> stencil_coefficients(int order) {
    float c[8] = {0};
    const int h = rtm_b200_stencil_coefficients(order, c);
    if (h < 0) throw std::runtime_error("unsupported spatial order (use 2, 4, 6, 8, 10 or 12)");
    return std::vector<float>(c, c + h + 1);
}

float ricker(float t, float f0) { return rtm_b200_ricker(t, f0); }

float max_stable_dt(float vmax, const Grid& g, int order) {
    const float dt = rtm_b200_max_stable_dt(vmax, g.dx, g.dz, order);
    if (dt < 0.0f) throw std::runtime_error("unsupported spatial order (use 2, 4, 6, 8, 10 or 12)");
    return dt;
}

float points_per_wavelength(float vmin, float f0, const Grid& g) {
    return rtm_b200_points_per_wavelength(vmin, f0, g.dx, g.dz);
}

void mute_direct_wave(ShotRecord& s, float v_surface, float t_pad, float t_taper) {
    rtm_b200_shot c{};
    c.sx = s.sx;
    c.sz = s.sz;
    c.nrec = s.nrec();
    c.nt = s.nt;
    c.dt = s.dt;
    c.rx = s.rx.data();
    c.rz = s.rz.data();
    rtm_b200_mute_direct_wave(&c, s.traces.data(), v_surface, t_pad, t_taper);
}

}  // namespace rtm_b200
