// comparison.cpp -- the image comparison metrics and the stack post-processing
// on the host.
//
// The metrics are the reference's parity tool (src/benchmark/comparison.cpp:7-35
// and the gate of src/tools/compare_main.cpp:52-53): every figure is a function
// of five running sums in double precision taken in index order, so the results
// here equal the reference's rtm_compare bit for bit.  The post-processing
// definitions are those of src/rtm/imaging.cpp:48-75 (float arithmetic in the
// same operation order, so the `_illum` / `_filtered` outputs are identical).
#include <algorithm>
#include <cmath>
#include <stdexcept>

#include "rtm_b200_engine.hpp"

namespace rtm_b200 {

namespace {

// One pass over (reference, test) pairs: the moments the metrics need.
struct Moments {
    double abs_err = 0;     // sum |r - t|
    double sq_err = 0;      // sum (r - t)^2
    double rr = 0, tt = 0;  // sum r^2, sum t^2
    double rt = 0;          // sum r t
    double worst = 0;       // max |r - t| (first index wins a tie)
    std::size_t at = 0;
    double r_peak = 0, t_peak = 0;

    void add(std::size_t i, double r, double t) {
        const double e = r - t;
        const double ae = std::fabs(e);
        if (ae > worst) {
            worst = ae;
            at = i;
        }
        abs_err += ae;
        sq_err += e * e;
        rr += r * r;
        tt += t * t;
        rt += r * t;
        r_peak = std::max(r_peak, std::fabs(r));
        t_peak = std::max(t_peak, std::fabs(t));
    }
};

double ratio_or_zero(double num, double den) { return den > 0 ? num / den : 0.0; }

}  // namespace

ImageDiff compare_images(const std::vector<float>& ref, const std::vector<float>& test) {
    if (ref.size() != test.size()) throw std::runtime_error("image size mismatch in comparison");
    ImageDiff out;
    out.n = ref.size();
    if (out.n == 0) return out;
    Moments m;
    for (std::size_t i = 0; i < out.n; ++i) m.add(i, ref[i], test[i]);
    const double n = (double)out.n;
    out.max_abs = m.worst;
    out.argmax = m.at;
    out.ref_max_abs = m.r_peak;
    out.test_max_abs = m.t_peak;
    out.mean_abs = m.abs_err / n;
    out.rms = std::sqrt(m.sq_err / n);
    out.l2_relative = m.rr > 0 ? std::sqrt(m.sq_err / m.rr) : 0.0;
    out.max_relative = ratio_or_zero(m.worst, m.r_peak);
    out.correlation = ratio_or_zero(m.rt, std::sqrt(m.rr * m.tt));
    return out;
}

bool gate_pass(const ImageDiff& d, double l2_max, double corr_min) {
    return d.l2_relative < l2_max && d.correlation > corr_min;
}

// image <- image / (S + eps_relative * max S + 1e-30): balances amplitudes and
// leaves reflector positions where they are.
void illumination_compensation(std::vector<float>& image, const std::vector<float>& illumination,
                               float eps_relative) {
    if (image.size() != illumination.size()) throw std::runtime_error("illumination size mismatch");
    const float peak = illumination.empty() ? 0.0f : *std::max_element(illumination.begin(), illumination.end());
    const float floor_term = eps_relative * std::max(peak, 0.0f) + 1e-30f;
    std::transform(image.begin(), image.end(), illumination.begin(), image.begin(),
                   [floor_term](float i, float s) { return i / (s + floor_term); });
}

// Second-difference high-pass (1/dx^2 d2/dx2 + 1/dz^2 d2/dz2) of the interior;
// the outermost rows and columns become zero.
void laplacian_filter(std::vector<float>& image, const Grid& g) {
    const float wx = 1.0f / (g.dx * g.dx);
    const float wz = 1.0f / (g.dz * g.dz);
    const std::size_t sx = (std::size_t)g.nz;   // neighbour offset along x (zfast)
    auto d2 = [&](std::size_t i, std::size_t s) { return image[i + s] - 2.0f * image[i] + image[i - s]; };
    std::vector<float> out(image.size(), 0.0f);
    for (int ix = 1; ix + 1 < g.nx; ++ix) {
        const std::size_t col = (std::size_t)ix * sx;
        for (int iz = 1; iz + 1 < g.nz; ++iz) {
            const std::size_t i = col + (std::size_t)iz;
            out[i] = wx * d2(i, sx) + wz * d2(i, 1);
        }
    }
    image.swap(out);
}

}  // namespace rtm_b200
