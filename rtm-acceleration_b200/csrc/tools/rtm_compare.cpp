// rtm_compare -- compare a test image with a reference image (raw float32):
// the reference's metrics and its default gate, L2rel < 1e-5 and
// correlation > 0.9999; exit status 0 on PASS, 2 on FAIL, 1 on error.
#include <cstdio>
#include <fstream>
#include <stdexcept>
#include <string>

#include "rtm_b200_engine.hpp"

using namespace rtm_b200;

int main(int argc, char** argv) try {
    if (argc < 3) {
        std::printf("usage: rtm_compare REFERENCE.bin TEST.bin [--nx N --nz N] [--csv PATH --engine NAME "
                    "--dataset NAME]\n");
        return 1;
    }
    const std::string ref_path = argv[1], test_path = argv[2];
    int nx = 0, nz = 0;
    std::string csv, engine = "unknown", dataset = "unknown";
    for (int i = 3; i < argc; ++i) {
        const std::string a = argv[i];
        if (a == "--nx" && i + 1 < argc) nx = std::stoi(argv[++i]);
        else if (a == "--nz" && i + 1 < argc) nz = std::stoi(argv[++i]);
        else if (a == "--csv" && i + 1 < argc) csv = argv[++i];
        else if (a == "--engine" && i + 1 < argc) engine = argv[++i];
        else if (a == "--dataset" && i + 1 < argc) dataset = argv[++i];
        else throw std::runtime_error("unknown option: " + a);
    }
    const auto ref = io::read_raw_floats(ref_path);
    const auto test = io::read_raw_floats(test_path);
    const ImageDiff d = compare_images(ref, test);
    std::printf("samples      %zu\nmax_abs      %.9g", d.n, d.max_abs);
    if (nx > 0 && nz > 0) std::printf("  at (ix %zu, iz %zu)", d.argmax / (size_t)nz, d.argmax % (size_t)nz);
    std::printf("\nmean_abs     %.9g\nrms          %.9g\nl2_relative  %.9g\nmax_relative %.9g\ncorrelation  %.12f\n",
                d.mean_abs, d.rms, d.l2_relative, d.max_relative, d.correlation);
    const bool pass = gate_pass(d);
    std::printf("gate: L2rel < 1e-05 and corr > 0.9999  =>  %s\n", pass ? "PASS" : "FAIL");
    if (!csv.empty()) {
        bool header = true;
        {
            std::ifstream e(csv);
            header = !(e && e.peek() != std::ifstream::traits_type::eof());
        }
        std::ofstream c(csv, std::ios::app);
        if (!c) throw std::runtime_error("cannot append compare csv: " + csv);
        if (header) c << "engine,dataset,max_abs,mean_abs,rms,l2_relative,max_relative,correlation,pass\n";
        c.precision(9);
        c << engine << ',' << dataset << ',' << d.max_abs << ',' << d.mean_abs << ',' << d.rms << ',' << d.l2_relative
          << ',' << d.max_relative << ',' << d.correlation << ',' << (pass ? 1 : 0) << '\n';
    }
    return pass ? 0 : 2;
} catch (const std::exception& e) {
    std::fprintf(stderr, "ERROR: %s\n", e.what());
    return 1;
}
