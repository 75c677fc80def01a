// comparison.cpp -- image comparison in double precision and the stack
// post-processing (reference src/benchmark/comparison.cpp:7-35 formulas and
// src/rtm/imaging.cpp:48-75 definitions, written here from those formulas).
#include <algorithm>
#include <cmath>
#include <stdexcept>

#include "rtm_b200_engine.hpp"

namespace rtm_b200 {

ImageDiff compare_images(const std::vector<float>& ref, const std::vector<float>& test) {
    if (ref.size() != test.size()) throw std::runtime_error("image size mismatch in comparison");
    ImageDiff d;
    d.n = ref.size();
    if (d.n == 0) return d;
    double sum_abs = 0, sum_sq = 0, ref_sq = 0, test_sq = 0, cross = 0;
    for (std::size_t i = 0; i < d.n; ++i) {
        const double a = ref[i], b = test[i], e = std::fabs(a - b);
        if (e > d.max_abs) { d.max_abs = e; d.argmax = i; }
        sum_abs += e;
        sum_sq += (a - b) * (a - b);
        ref_sq += a * a;
        test_sq += b * b;
        cross += a * b;
        d.ref_max_abs = std::max(d.ref_max_abs, std::fabs(a));
        d.test_max_abs = std::max(d.test_max_abs, std::fabs(b));
    }
    d.mean_abs = sum_abs / (double)d.n;
    d.rms = std::sqrt(sum_sq / (double)d.n);
    d.l2_relative = ref_sq > 0 ? std::sqrt(sum_sq / ref_sq) : 0.0;
    d.max_relative = d.ref_max_abs > 0 ? d.max_abs / d.ref_max_abs : 0.0;
    const double den = std::sqrt(ref_sq * test_sq);
    d.correlation = den > 0 ? cross / den : 0.0;
    return d;
}

bool gate_pass(const ImageDiff& d, double l2_max, double corr_min) {
    return d.l2_relative < l2_max && d.correlation > corr_min;
}

// I / (S + eps * max S): balances amplitudes, leaves reflector positions.
void illumination_compensation(std::vector<float>& image, const std::vector<float>& illumination,
                               float eps_relative) {
    if (image.size() != illumination.size()) throw std::runtime_error("illumination size mismatch");
    float smax = 0.0f;
    for (float s : illumination) smax = std::max(smax, s);
    const float eps = eps_relative * smax + 1e-30f;
    for (std::size_t i = 0; i < image.size(); ++i) image[i] /= (illumination[i] + eps);
}

// Five-point Laplacian high-pass on the interior; the border becomes zero.
void laplacian_filter(std::vector<float>& image, const Grid& g) {
    std::vector<float> out(image.size(), 0.0f);
    const float ax = 1.0f / (g.dx * g.dx), az = 1.0f / (g.dz * g.dz);
    for (int ix = 1; ix + 1 < g.nx; ++ix)
        for (int iz = 1; iz + 1 < g.nz; ++iz) {
            const std::size_t i = (std::size_t)ix * g.nz + iz;
            out[i] = ax * (image[i + g.nz] - 2.0f * image[i] + image[i - g.nz]) +
                     az * (image[i + 1] - 2.0f * image[i] + image[i - 1]);
        }
    image.swap(out);
}

}  // namespace rtm_b200
