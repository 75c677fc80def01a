// engine_b200.cpp -- B200RTM: the RTMEngine interface over librtm_b200.so.
#include <stdexcept>
#include <string>

#include "rtm_b200_engine.hpp"

namespace rtm_b200 {
namespace {

rtm_b200_shot to_c(const ShotRecord& s) {
    rtm_b200_shot c{};
    c.sx = s.sx;
    c.sz = s.sz;
    c.nrec = s.nrec();
    c.nt = s.nt;
    c.dt = s.dt;
    c.rx = s.rx.data();
    c.rz = s.rz.data();
    c.traces = s.traces.empty() ? nullptr : s.traces.data();
    c.window_x0 = s.window_x0;
    c.window_nx = s.window_nx;
    return c;
}

}  // namespace

B200RTM::B200RTM(const B200Options& opt) : opt_(opt) {}

B200RTM::~B200RTM() {
    if (h_) rtm_b200_destroy(h_);
}

const char* B200RTM::name() const {
    switch (opt_.mode) {
        case RTM_B200_MODE_BATCH: return "b200-batch";
        case RTM_B200_MODE_SERVE: return "b200-serve";
        default: return "b200";
    }
}

void B200RTM::check(int rc, const char* what) const {
    if (rc == RTM_B200_OK) return;
    char buf[1024] = {0};
    rtm_b200_last_error(h_, buf, sizeof buf);
    throw std::runtime_error(std::string(what) + ": " + buf);
}

void B200RTM::copy_times() {
    rtm_b200_times t{};
    if (h_ && rtm_b200_get_times(h_, &t) == RTM_B200_OK) {
        times.total = t.total;
        times.h2d = t.h2d;
        times.kernel = t.kernel;
        times.d2h = t.d2h;
    }
}

rtm_b200_times B200RTM::raw_times() const {
    rtm_b200_times t{};
    if (h_) rtm_b200_get_times(h_, &t);
    return t;
}

void B200RTM::setup(const VelocityModel& model, const RTMParams& par, const TimeAxis& ta) {
    if (h_) {
        rtm_b200_destroy(h_);
        h_ = nullptr;
    }
    rtm_b200_config cfg;
    rtm_b200_config_init(&cfg);
    cfg.mode = opt_.mode;
    cfg.device = opt_.device;
    cfg.nb = par.nb;
    cfg.order = par.order;
    cfg.sponge_alpha = par.sponge_alpha;
    cfg.store_interval = par.store_interval;
    cfg.f0 = par.f0;
    cfg.verbose = par.verbose ? 1 : 0;
    cfg.snap_precision = opt_.snap_precision;
    cfg.arithmetic = opt_.arithmetic;
    cfg.accumulation = opt_.accumulation;
    cfg.max_shots_in_flight = opt_.max_shots_in_flight;
    cfg.tile_cols = opt_.tile_cols;
    check(rtm_b200_create(&cfg, &h_), "rtm_b200_create");
    const Grid& g = model.grid;
    check(rtm_b200_setup(h_, model.v.data(), g.nx, g.nz, g.dx, g.dz, g.ox, g.oz, ta.nt, ta.dt), "setup");
    g_ = g;
    g_.nb = par.nb;
    par_ = par;
    ta_ = ta;
    nsnap_ = rtm_b200_num_snapshots(h_);
}

void B200RTM::migrate(const std::vector<ShotRecord>& shots, std::vector<float>& image,
                      std::vector<float>& illumination) {
    if (!h_) throw std::runtime_error("migrate before setup");
    std::vector<rtm_b200_shot> c;
    c.reserve(shots.size());
    for (const auto& s : shots) c.push_back(to_c(s));
    image.assign(g_.n_interior(), 0.0f);
    illumination.assign(g_.n_interior(), 0.0f);
    rtm_b200_reset_times(h_);
    check(rtm_b200_migrate(h_, c.data(), (int)c.size(), image.data(), illumination.data()), "migrate");
    copy_times();
}

void B200RTM::postprocess(float eps_relative, bool compensate_filtered, std::vector<float>* illum_out,
                          std::vector<float>* filtered_out) {
    if (!h_) throw std::runtime_error("postprocess before setup");
    if (illum_out) illum_out->assign(g_.n_interior(), 0.0f);
    if (filtered_out) filtered_out->assign(g_.n_interior(), 0.0f);
    check(rtm_b200_postprocess(h_, eps_relative, compensate_filtered ? 1 : 0, illum_out ? illum_out->data() : nullptr,
                               filtered_out ? filtered_out->data() : nullptr),
          "postprocess");
}

void B200RTM::forward_propagation(const ShotRecord& shot, std::vector<float>* snapshots,
                                  std::vector<float>* recorded) {
    if (!h_) throw std::runtime_error("forward_propagation before setup");
    const rtm_b200_shot c = to_c(shot);
    if (snapshots) snapshots->assign((std::size_t)nsnap_ * g_.n_interior(), 0.0f);
    if (recorded) recorded->assign((std::size_t)shot.nrec() * ta_.nt, 0.0f);
    check(rtm_b200_forward(h_, &c, snapshots ? snapshots->data() : nullptr, recorded ? recorded->data() : nullptr),
          "forward_propagation");
}

void B200RTM::backward_propagation(const ShotRecord& shot, const std::vector<float>& snapshots,
                                   std::vector<float>& image, std::vector<float>& illumination) {
    if (!h_) throw std::runtime_error("backward_propagation before setup");
    const rtm_b200_shot c = to_c(shot);
    image.resize(g_.n_interior(), 0.0f);
    illumination.resize(g_.n_interior(), 0.0f);
    check(rtm_b200_backward(h_, &c, snapshots.empty() ? nullptr : snapshots.data(), image.data(),
                            illumination.data()),
          "backward_propagation");
}

void B200RTM::imaging(const float* fwd_snapshot, const float* bwd_extended, std::vector<float>& image,
                      std::vector<float>& illumination) {
    if (!h_) throw std::runtime_error("imaging before setup");
    image.resize(g_.n_interior(), 0.0f);
    illumination.resize(g_.n_interior(), 0.0f);
    check(rtm_b200_imaging(h_, fwd_snapshot, bwd_extended, image.data(), illumination.data()), "imaging");
}

void B200RTM::model_shot(ShotRecord& shot) {
    std::vector<ShotRecord> one(1, shot);
    model_shots(one);
    shot = std::move(one[0]);
}

void B200RTM::model_shots(std::vector<ShotRecord>& shots) {
    if (!h_) throw std::runtime_error("model_shot before setup");
    std::vector<rtm_b200_shot> c;
    std::size_t total = 0;
    for (const auto& s : shots) {
        c.push_back(to_c(s));
        c.back().traces = nullptr;
        total += (std::size_t)s.nrec() * ta_.nt;
    }
    std::vector<float> out(total > 0 ? total : 1);
    check(rtm_b200_model_shots(h_, c.data(), (int)c.size(), out.data()), "model_shot");
    std::size_t off = 0;
    for (auto& s : shots) {
        const std::size_t n = (std::size_t)s.nrec() * ta_.nt;
        s.traces.assign(out.begin() + (long)off, out.begin() + (long)(off + n));
        s.nt = ta_.nt;
        s.dt = ta_.dt;
        off += n;
    }
}

std::string B200RTM::device_name() const {
    char b[256] = {0};
    if (h_) rtm_b200_device_name(h_, b, sizeof b);
    return b;
}

}  // namespace rtm_b200
