// rtm -- command-line migration with the B200 engines.  Same flags, defaults,
// precedence and outputs as the reference's `rtm` (src/main.cpp): a velocity
// model (raw float32 + .hdr sidecar, CLI values win), shots (RTMS or SEG-Y),
// optional direct-wave mute, and the raw zero-lag image image[ix*nz+iz] as the
// main output, plus the optional _illummap / _illum / _filtered files.
// Engine-specific options: --snap-precision, --arith, --max-in-flight,
// --tile-cols; --check-inputs reads and validates the inputs only.
#include <chrono>
#include <cstdio>
#include <fstream>
#include <stdexcept>
#include <string>

#include "options.hpp"
#include "rtm_b200_engine.hpp"

using namespace rtm_b200;

static void usage() {
    std::printf(
        "rtm -- 2D acoustic reverse time migration on one B200 GPU\n\n"
        "  --engine NAME          b200 | b200-batch | b200-serve      (default b200)\n"
        "  --list-engines         print the engine names and exit\n"
        "  --gpus N               must be 1\n"
        "  --velocity PATH        float32 velocity model (m/s)          [required]\n"
        "  --shots PATH           .bin (RTMS) or .sgy/.segy shot file    [required]\n"
        "  --output PATH          migrated image, float32, image[ix*nz+iz] [required]\n"
        "  --vel-header PATH      header file (default: <velocity>.hdr)\n"
        "  --nx N --nz N --dx M --dz M --ox M --oz M --vel-layout zfast|xfast\n"
        "  --order N (8)  --nb N (60)  --sponge-alpha F (0.0053)  --f0 F (12)\n"
        "  --store-interval N (1)  --nt N  --max-shots N  --mute-direct V (0 = off)\n"
        "  --illumination  --filter laplacian  --write-illum-map\n"
        "  --benchmark PATH  --benchmark-csv PATH  --dataset NAME\n"
        "  --segy-src-depth M (10)  --segy-rec-depth M (10)  --quiet\n"
        "  --snap-precision f32|bf16|f16|recon  --arith auto|ieee|fma|fp64  --max-in-flight N  --tile-cols 0|16|32\n"
        "  --check-inputs         read and validate the inputs, print a summary, exit\n");
}

// Which velocity-header fields were set on the command line; those win over the
// sidecar header.
struct GivenHeaderFields {
    bool nx = false, nz = false, dx = false, dz = false, ox = false, oz = false, layout = false;
};

int main(int argc, char** argv) try {
    std::string vel_path, shots_path, out_path, hdr_path, filter = "none", engine_name = "b200";
    std::string bench_path, bench_csv, dataset;
    io::VelocityHeader vh;
    GivenHeaderFields given;
    RTMParams par;
    B200Options opt;
    int gpus = 1, nt_override = 0, max_shots = 0;
    bool want_illum = false, want_map = false, check_only = false;
    float mute_v = 0.0f, segy_sz = 10.0f, segy_rz = 10.0f;

    cli::Options table;
    table.text("--velocity", vel_path).text("--shots", shots_path).text("--output", out_path)
        .text("--vel-header", hdr_path)
        .integer("--nx", vh.nx, &given.nx).integer("--nz", vh.nz, &given.nz)
        .real("--dx", vh.dx, &given.dx).real("--dz", vh.dz, &given.dz)
        .real("--ox", vh.ox, &given.ox).real("--oz", vh.oz, &given.oz)
        .text("--vel-layout", vh.layout, &given.layout)
        .integer("--order", par.order).integer("--nb", par.nb).real("--sponge-alpha", par.sponge_alpha)
        .real("--f0", par.f0).integer("--store-interval", par.store_interval)
        .integer("--nt", nt_override).integer("--max-shots", max_shots).real("--mute-direct", mute_v)
        .boolean("--illumination", want_illum).boolean("--write-illum-map", want_map).text("--filter", filter)
        .text("--benchmark", bench_path).text("--benchmark-csv", bench_csv).text("--dataset", dataset)
        .real("--segy-src-depth", segy_sz).real("--segy-rec-depth", segy_rz)
        .boolean("--quiet", par.verbose, false)
        .text("--engine", engine_name).integer("--gpus", gpus)
        .choice("--snap-precision", opt.snap_precision,
                {{"f32", RTM_B200_SNAP_F32}, {"bf16", RTM_B200_SNAP_BF16}, {"f16", RTM_B200_SNAP_F16},
                 {"recon", RTM_B200_SNAP_RECON}})
        .choice("--arith", opt.arithmetic,
                {{"auto", RTM_B200_ARITH_AUTO}, {"ieee", RTM_B200_ARITH_IEEE}, {"fma", RTM_B200_ARITH_FMA},
                 {"fp64", RTM_B200_ARITH_FP64}})
        .integer("--max-in-flight", opt.max_shots_in_flight).integer("--tile-cols", opt.tile_cols)
        .boolean("--check-inputs", check_only)
        .terminal("--list-engines").terminal("--help").terminal("-h");
    const std::string stop = table.parse(argc, argv);
    if (stop == "--list-engines") {
        for (const auto& n : list_engines()) std::printf("%s\n", n.c_str());
        return 0;
    }
    if (!stop.empty()) { usage(); return 0; }
    if (vel_path.empty() || shots_path.empty() || (out_path.empty() && !check_only)) {
        usage();
        throw std::runtime_error("--velocity, --shots and --output are required");
    }
    std::unique_ptr<RTMEngine> engine = make_engine(engine_name, gpus, &opt);
    const auto t0 = std::chrono::steady_clock::now();

    // Header precedence: explicit CLI values, then --vel-header, then <velocity>.hdr.
    io::VelocityHeader side;
    bool found = false;
    if (!hdr_path.empty()) {
        if (!io::read_header_file(hdr_path, side)) throw std::runtime_error("cannot read velocity header: " + hdr_path);
        found = true;
    } else {
        found = io::read_header_file(vel_path + ".hdr", side);
    }
    if (found) {
        const io::VelocityHeader cli_values = vh;
        vh = side;
        if (given.nx) vh.nx = cli_values.nx;
        if (given.nz) vh.nz = cli_values.nz;
        if (given.dx) vh.dx = cli_values.dx;
        if (given.dz) vh.dz = cli_values.dz;
        if (given.ox) vh.ox = cli_values.ox;
        if (given.oz) vh.oz = cli_values.oz;
        if (given.layout) vh.layout = cli_values.layout;
    }
    VelocityModel model = io::read_velocity_raw(vel_path, vh);
    std::vector<ShotRecord> shots = io::read_shots(shots_path, segy_sz, segy_rz);
    if (max_shots > 0 && (int)shots.size() > max_shots) shots.resize((std::size_t)max_shots);
    if (mute_v > 0.0f)
        for (auto& s : shots) mute_direct_wave(s, mute_v, 1.0f / par.f0, 1.0f / par.f0);
    engine->times.io = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();

    TimeAxis ta;
    ta.nt = nt_override > 0 ? std::min(nt_override, shots[0].nt) : shots[0].nt;
    ta.dt = shots[0].dt;
    const float dt_max = max_stable_dt(model.vmax(), model.grid, par.order);
    const float ppw = points_per_wavelength(model.vmin(), par.f0, model.grid);
    if (check_only) {
        double sum = 0.0;
        for (const auto& s : shots)
            for (float v : s.traces) sum += v;
        std::printf("{\"nx\": %d, \"nz\": %d, \"dx\": %g, \"dz\": %g, \"ox\": %g, \"oz\": %g, \"vmin\": %g, "
                    "\"vmax\": %g, \"shots\": %zu, \"nrec\": %d, \"nt\": %d, \"dt\": %.9g, \"dt_max\": %.9g, "
                    "\"ppw\": %g, \"trace_sum\": %.17g, \"sx0\": %.9g}\n",
                    model.grid.nx, model.grid.nz, model.grid.dx, model.grid.dz, model.grid.ox, model.grid.oz,
                    model.vmin(), model.vmax(), shots.size(), shots[0].nrec(), ta.nt, ta.dt, dt_max, ppw, sum,
                    shots[0].sx);
        return 0;
    }

    engine->setup(model, par, ta);
    const Grid& g = engine->grid();
    if (par.verbose)
        std::printf("\n=== MODEL ===\n  nx = %d, nz = %d, dx = %.2f m, dz = %.2f m\n  vmin = %.1f, vmax = %.1f m/s\n"
                    "  nt = %d, dt = %.6f s\n  order = %d, nb = %d, f0 = %.2f Hz, store_interval = %d\n"
                    "  shots = %zu, receivers/shot = %d\n  CFL: dt = %.6f s, dt_max = %.6f s %s\n"
                    "  Dispersion: %.2f points per shortest wavelength %s\n  Snapshot memory: %.1f MiB\n"
                    "  Device: %s\n\n",
                    g.nx, g.nz, g.dx, g.dz, model.vmin(), model.vmax(), ta.nt, ta.dt, par.order, par.nb, par.f0,
                    par.store_interval, shots.size(), shots[0].nrec(), ta.dt, dt_max,
                    ta.dt <= dt_max ? "OK" : "*** UNSTABLE ***", ppw, ppw >= 4.0f ? "OK" : "*** DISPERSIVE ***",
                    engine->snapshot_bytes() / (1024.0 * 1024.0), engine->device_name().c_str());
    if (ta.dt > dt_max)
        throw std::runtime_error("time step violates the CFL condition -- reduce dt, reduce the FD order, or coarsen "
                                 "f0/dx");
    if (ppw < 3.0f)
        std::fprintf(stderr, "WARNING: fewer than 3 points per wavelength; the image will be visibly dispersive.\n");

    std::vector<float> image, illum;
    if (par.verbose) std::printf("=== MIGRATION (%s) ===\n", engine->name());
    engine->migrate(shots, image, illum);
    io::write_raw_floats(out_path, image);
    if (par.verbose) std::printf("wrote %s  (%d x %d float32, image[ix*nz+iz])\n", out_path.c_str(), g.nx, g.nz);
    const auto dot = out_path.find_last_of('.');
    const std::string stem = dot == std::string::npos ? out_path : out_path.substr(0, dot);
    if (want_map) io::write_raw_floats(stem + "_illummap.bin", illum);
    // _illum and _filtered (reference src/main.cpp:211-223): computed on the
    // device from the stack the migration left there for the B200 engines, on
    // the host otherwise.
    auto* b200 = dynamic_cast<B200RTM*>(engine.get());
    if (b200 && (want_illum || filter == "laplacian")) {
        std::vector<float> ti, tf;
        b200->postprocess(1e-4f, want_illum, want_illum ? &ti : nullptr, filter == "laplacian" ? &tf : nullptr);
        if (want_illum) io::write_raw_floats(stem + "_illum.bin", ti);
        if (filter == "laplacian") io::write_raw_floats(stem + "_filtered.bin", tf);
    } else {
        if (want_illum) {
            std::vector<float> t = image;
            illumination_compensation(t, illum, 1e-4f);
            io::write_raw_floats(stem + "_illum.bin", t);
        }
        if (filter == "laplacian") {
            std::vector<float> t = image;
            if (want_illum) illumination_compensation(t, illum, 1e-4f);
            laplacian_filter(t, g);
            io::write_raw_floats(stem + "_filtered.bin", t);
        }
    }

    // Report: the reference's cell-update convention (2 nt N_ext per shot).
    const double upd = 2.0 * ta.nt * (double)g.nxe() * g.nze() * (double)shots.size();
    const double sec = engine->times.total > 0 ? engine->times.total : 1e-30;
    char line[512];
    std::snprintf(line, sizeof line,
                  "engine %s | device %s | shots %zu | total %.3f s | kernel %.3f s | h2d %.3f s | d2h %.3f s | "
                  "%.3f G cell updates/s | %.2f shots/s\n",
                  engine->name(), engine->device_name().c_str(), shots.size(), engine->times.total,
                  engine->times.kernel, engine->times.h2d, engine->times.d2h, upd / sec / 1e9, shots.size() / sec);
    if (par.verbose) std::printf("\n%s", line);
    if (!bench_path.empty()) std::ofstream(bench_path, std::ios::app) << line;
    if (!bench_csv.empty()) {
        bool header = true;
        {
            std::ifstream e(bench_csv);
            header = !(e && e.peek() != std::ifstream::traits_type::eof());
        }
        std::ofstream c(bench_csv, std::ios::app);
        if (header) c << "engine,device,dataset,nx,nz,nb,order,nt,shots,total_s,kernel_s,gcell_updates_per_s\n";
        c << engine->name() << ',' << engine->device_name() << ',' << dataset << ',' << g.nx << ',' << g.nz << ','
          << g.nb << ',' << par.order << ',' << ta.nt << ',' << shots.size() << ',' << engine->times.total << ','
          << engine->times.kernel << ',' << upd / sec / 1e9 << '\n';
    }
    return 0;
} catch (const std::exception& e) {
    std::fprintf(stderr, "ERROR: %s\n", e.what());
    return 1;
}
