// numerics.cpp -- see numerics.hpp.
#include "numerics.hpp"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <numeric>

namespace rtmb {

int stencil_half(int order) {
    if (order < 2 || order > 2 * kMaxHalf || (order % 2) != 0) return -1;
    return order / 2;
}

namespace {
int64_t factorial(int n) {
    int64_t f = 1;
    for (int i = 2; i <= n; ++i) f *= i;
    return f;
}
float ratio_to_float(int64_t num, int64_t den) {
    const int64_t g = std::gcd(num < 0 ? -num : num, den);
    num /= g;
    den /= g;
    // |num|, den < 2^24 for every order <= 12, so both convert exactly and the
    // IEEE quotient is the correctly rounded value of the rational.
    return (float)num / (float)den;
}
}  // namespace

bool stencil_coefficients(int order, float* c) {
    const int M = stencil_half(order);
    if (M < 0) return false;
    const int64_t fm = factorial(M);
    for (int k = 1; k <= M; ++k) {
        const int64_t num = 2 * fm * fm * ((k % 2) ? 1 : -1);
        const int64_t den = (int64_t)k * k * factorial(M - k) * factorial(M + k);
        c[k] = ratio_to_float(num, den);
    }
    int64_t L = 1;
    for (int k = 1; k <= M; ++k) L = std::lcm(L, (int64_t)k * k);
    int64_t s = 0;
    for (int k = 1; k <= M; ++k) s += L / ((int64_t)k * k);
    c[0] = ratio_to_float(-2 * s, L);
    return true;
}

float stencil_abs_sum(int order) {
    float c[kMaxHalf + 1];
    if (!stencil_coefficients(order, c)) return -1.0f;
    const int h = order / 2;
    float s = std::fabs(c[0]);
    for (int k = 1; k <= h; ++k) s += 2.0f * std::fabs(c[k]);
    return s;
}

float ricker(float t, float f0) {
    const float a = (float)(M_PI * M_PI) * f0 * f0 * t * t;
    return (1.0f - 2.0f * a) * std::exp(-a);
}

float max_stable_dt(float vmax, float dx, float dz, int order) {
    const float S = stencil_abs_sum(order);
    return 2.0f / (vmax * std::sqrt(S * (1.0f / (dx * dx) + 1.0f / (dz * dz))));
}

float points_per_wavelength(float vmin, float f0, float dx, float dz) {
    const float fmax = 2.5f * f0;
    const float lambda_min = vmin / fmax;
    return lambda_min / std::max(dx, dz);
}

float cerjan_taper(int i, int n, int nb, float alpha) {
    const int d = std::min(i, n - 1 - i);
    if (d >= nb) return 1.0f;
    const float a = alpha * (float)(nb - d);
    return std::exp(-a * a);
}

std::vector<float> ricker_wavelet(int nt, float dt, float f0) {
    std::vector<float> w((size_t)std::max(nt, 0));
    const float t0 = 1.2f / f0;
    for (int it = 0; it < nt; ++it) w[(size_t)it] = ricker((float)it * dt - t0, f0);
    return w;
}

ScaledCoefficients scaled_coefficients(int order, float dx, float dz) {
    ScaledCoefficients s;
    float c[kMaxHalf + 1] = {};
    if (!stencil_coefficients(order, c)) return s;
    const int h = order / 2;
    const float idx2 = 1.0f / (dx * dx);
    const float idz2 = 1.0f / (dz * dz);
    s.c0 = c[0] * (idx2 + idz2);
    for (int k = 1; k <= h; ++k) {
        s.cx[k] = c[k] * idx2;
        s.cz[k] = c[k] * idz2;
    }
    return s;
}

GridDims make_grid(int nx, int nz, int nb, int half) {
    GridDims g;
    g.nx = nx; g.nz = nz; g.nb = nb; g.half = half;
    g.nxe = nx + 2 * nb;
    g.nze = nz + 2 * nb;
    g.ldz = (g.nze + 7) & ~7;
    g.zs0 = nb & ~3;
    g.lds = ((nb + nz + 3) & ~3) - g.zs0;
    g.ntz = (g.nze + kTileZ - 1) / kTileZ;
    return g;
}

}  // namespace rtmb
