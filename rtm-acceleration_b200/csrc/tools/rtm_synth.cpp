// rtm_synth -- synthetic shot gathers modelled on the GPU with the migration's
// own propagator.  Same flags and defaults as the reference's generator
// (src/tools/make_synthetic.cpp): a three-layer model whose second interface
// dips (slope 0.15 about the centre) with a 60 x 60 m 2800 m/s box at
// (1200, 700) m, or an existing velocity model; a split-spread surface line of
// nrec = (nx-1) dx / rec_dx + 1 live receivers; shots at xmax (is+1)/(nshots+1)
// or x0 + is dx; output in RTMS format.  All shots are modelled in one batched
// call; the traces equal the reference's modelling bit for bit (plain IEEE
// arithmetic).
#include <chrono>
#include <cstdio>
#include <stdexcept>
#include <string>

#include "options.hpp"
#include "rtm_b200_engine.hpp"

using namespace rtm_b200;

int main(int argc, char** argv) try {
    std::string outdir = "data/synthetic", vel_path, shots_out, engine_name = "b200-batch";
    int nx = 201, nz = 151, nt = 1400, nshots = 4, order = 8, nb = 60;
    float dx = 10.0f, dz = 10.0f, dt = 0.001f, f0 = 12.0f, src_z = 20.0f, rec_z = 20.0f, rec_dx = 20.0f;
    float shot_x0 = -1.0f, shot_dx = -1.0f;
    io::VelocityHeader vh;
    bool given_nx = false, given_nz = false, given_dx = false, given_dz = false;
    cli::Options table;
    table.text("--outdir", outdir)
        .integer("--nx", nx, &given_nx).integer("--nz", nz, &given_nz)
        .real("--dx", dx, &given_dx).real("--dz", dz, &given_dz)
        .integer("--nt", nt).real("--dt", dt).real("--f0", f0).integer("--nshots", nshots)
        .integer("--order", order).integer("--nb", nb)
        .real("--rec-dx", rec_dx).real("--src-z", src_z).real("--rec-z", rec_z)
        .text("--velocity", vel_path).text("--vel-layout", vh.layout).text("--shots-out", shots_out)
        .real("--shot-x0", shot_x0).real("--shot-dx", shot_dx).text("--engine", engine_name);
    table.parse(argc, argv);
    VelocityModel model;
    if (!vel_path.empty()) {
        io::VelocityHeader side;
        if (io::read_header_file(vel_path + ".hdr", side)) {
            // Sizes on the command line win.  The sidecar's layout applies unless
            // the command line asked for a layout other than the default zfast,
            // and its origin always applies.
            nx = given_nx ? nx : side.nx;
            nz = given_nz ? nz : side.nz;
            dx = given_dx ? dx : side.dx;
            dz = given_dz ? dz : side.dz;
            if (vh.layout == "zfast") vh.layout = side.layout;
            vh.ox = side.ox;
            vh.oz = side.oz;
        }
        vh.nx = nx; vh.nz = nz; vh.dx = dx; vh.dz = dz;
        model = io::read_velocity_raw(vel_path, vh);
    } else {
        Grid& g = model.grid;
        g.nx = nx; g.nz = nz; g.dx = dx; g.dz = dz;
        model.v.assign((size_t)nx * nz, 1500.0f);
        for (int ix = 0; ix < nx; ++ix) {
            const float x = ix * dx;
            const float zdip = 900.0f + 0.15f * (x - 0.5f * nx * dx);
            for (int iz = 0; iz < nz; ++iz) {
                const float z = iz * dz;
                float v = z >= 400.0f ? 2000.0f : 1500.0f;
                if (z >= zdip) v = 2500.0f;
                if (x >= 1200.0f && x < 1260.0f && z >= 700.0f && z < 760.0f) v = 2800.0f;
                model.v[(size_t)ix * nz + iz] = v;
            }
        }
        vh.nx = nx; vh.nz = nz; vh.dx = dx; vh.dz = dz; vh.ox = 0; vh.oz = 0; vh.layout = "zfast";
        io::write_velocity_raw(outdir + "/velocity.bin", model);
        io::write_header_file(outdir + "/velocity.bin.hdr", vh);
    }
    const int nrec = (int)((nx - 1) * dx / rec_dx) + 1;
    const float xmax = (nx - 1) * dx;
    std::vector<ShotRecord> shots((size_t)nshots);
    for (int is = 0; is < nshots; ++is) {
        ShotRecord& s = shots[(size_t)is];
        s.sx = shot_dx > 0.0f ? (shot_x0 >= 0.0f ? shot_x0 : 0.0f) + shot_dx * (float)is
                              : xmax * (float)(is + 1) / (float)(nshots + 1);
        s.sz = src_z;
        s.nt = nt;
        s.dt = dt;
        s.rx.resize((size_t)nrec);
        s.rz.assign((size_t)nrec, rec_z);
        for (int ir = 0; ir < nrec; ++ir) s.rx[(size_t)ir] = ir * rec_dx;
    }
    RTMParams par;
    par.nb = nb; par.order = order; par.f0 = f0; par.store_interval = 1;
    TimeAxis ta;
    ta.nt = nt; ta.dt = dt;
    auto engine = make_engine(engine_name);
    engine->setup(model, par, ta);
    const float dt_max = max_stable_dt(model.vmax(), engine->grid(), order);
    std::printf("modelling %d shots x %d receivers x %d samples on %d x %d cells (%s, %s); dt %.6f s, max stable %.6f s\n",
                nshots, nrec, nt, nx, nz, engine->name(), engine->device_name().c_str(), dt, dt_max);
    if (dt > dt_max) throw std::runtime_error("chosen dt is unstable");
    const auto t0 = std::chrono::steady_clock::now();
    static_cast<B200RTM*>(engine.get())->model_shots(shots);
    const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    const std::string path = shots_out.empty() ? outdir + "/shots.bin" : shots_out;
    io::write_shots_raw(path, shots);
    std::printf("modelling took %.3f s; wrote %s\n", sec, path.c_str());
    return 0;
} catch (const std::exception& e) {
    std::fprintf(stderr, "ERROR: %s\n", e.what());
    return 1;
}
