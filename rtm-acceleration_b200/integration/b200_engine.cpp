// b200_engine.cpp -- the B200 engine as one more rtm::RTMEngine of the
// reference code base (Marouane-Djabri/RTM-Acceleration, include/rtm_engine.hpp:20-83).
//
// This is the binding a maintainer of the reference adds as src/b200/: it is
// compiled against the reference's own headers and links librtm_b200.so through
// its C ABI (include/rtm_b200.h of this repository).  Each RTMEngine virtual
// maps onto one C entry point; a non-zero status becomes std::runtime_error,
// as everywhere in the reference.  oracle/Makefile (target ref-b200) builds the
// reference's unmodified CLI (src/main.cpp) with this engine registered by
// factory_b200.cpp, and tests/test_gpu_reference_binding.py runs it.
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "rtm_b200.h"
#include "rtm_engine.hpp"

namespace rtm {

class B200RTM : public RTMEngine {
public:
    explicit B200RTM(int mode) {
        rtm_b200_config_init(&cfg_);
        cfg_.mode = mode;   // RTM_B200_MODE_PLAIN / _BATCH / _SERVE
    }
    ~B200RTM() override {
        if (h_) rtm_b200_destroy(h_);
    }
    const char* name() const override {
        return cfg_.mode == RTM_B200_MODE_PLAIN ? "b200" : cfg_.mode == RTM_B200_MODE_BATCH ? "b200-batch" : "b200-serve";
    }

    void setup(const VelocityModel& m, const RTMParams& p, const TimeAxis& ta) override {
        if (h_) { rtm_b200_destroy(h_); h_ = nullptr; }
        cfg_.nb = p.nb; cfg_.order = p.order; cfg_.sponge_alpha = p.sponge_alpha;
        cfg_.store_interval = p.store_interval; cfg_.f0 = p.f0; cfg_.verbose = p.verbose ? 1 : 0;
        check(rtm_b200_create(&cfg_, &h_));
        const Grid& g = m.grid;
        check(rtm_b200_setup(h_, m.v.data(), g.nx, g.nz, g.dx, g.dz, g.ox, g.oz, ta.nt, ta.dt));
        g_ = g;
        g_.nb = p.nb;
        g_.half = p.order / 2;
        par_ = p;
        ta_ = ta;
        nsnap_ = rtm_b200_num_snapshots(h_);
    }

    void migrate(const std::vector<ShotRecord>& shots, std::vector<float>& image,
                 std::vector<float>& illum) override {
        std::vector<rtm_b200_shot> c = to_c(shots);
        image.assign(g_.n_interior(), 0.0f);   // assigned, like the reference's default migrate
        illum.assign(g_.n_interior(), 0.0f);
        rtm_b200_reset_times(h_);
        check(rtm_b200_migrate(h_, c.data(), (int)c.size(), image.data(), illum.data()));
        rtm_b200_times t{};
        rtm_b200_get_times(h_, &t);
        times.total = t.total; times.forward = t.forward; times.backward = t.backward;
        times.kernel = t.kernel; times.h2d = t.h2d; times.d2h = t.d2h;
    }

    void forward_propagation(const ShotRecord& s, std::vector<float>* snaps, std::vector<float>* rec) override {
        rtm_b200_shot c = to_c1(s);
        if (snaps) snaps->assign((size_t)nsnap_ * g_.n_interior(), 0.0f);
        if (rec) rec->assign((size_t)s.nrec() * ta_.nt, 0.0f);
        check(rtm_b200_forward(h_, &c, snaps ? snaps->data() : nullptr, rec ? rec->data() : nullptr));
    }
    void backward_propagation(const ShotRecord& s, const std::vector<float>& snaps, std::vector<float>& image,
                              std::vector<float>& illum) override {
        rtm_b200_shot c = to_c1(s);
        check(rtm_b200_backward(h_, &c, snaps.empty() ? nullptr : snaps.data(), image.data(), illum.data()));
    }
    void imaging(const float* f, const float* b, std::vector<float>& image, std::vector<float>& illum) override {
        check(rtm_b200_imaging(h_, f, b, image.data(), illum.data()));
    }
    void model_shot(ShotRecord& s) override {
        rtm_b200_shot c = to_c1(s);
        s.traces.assign((size_t)s.nrec() * ta_.nt, 0.0f);
        check(rtm_b200_model_shots(h_, &c, 1, s.traces.data()));
        s.nt = ta_.nt;
        s.dt = ta_.dt;
    }

    int num_devices() const override { return 1; }
    bool is_gpu() const override { return true; }
    std::string device_name() const override {
        char b[256] = {0};
        if (h_) rtm_b200_device_name(h_, b, sizeof b);
        return b;
    }

private:
    void check(int rc) const {
        if (rc == RTM_B200_OK) return;
        char b[1024] = {0};
        rtm_b200_last_error(h_, b, sizeof b);
        throw std::runtime_error(std::string("b200 engine: ") + b);
    }
    static rtm_b200_shot to_c1(const ShotRecord& s) {
        rtm_b200_shot c{};
        c.sx = s.sx; c.sz = s.sz; c.nrec = s.nrec(); c.nt = s.nt; c.dt = s.dt;
        c.rx = s.rx.data(); c.rz = s.rz.data();
        c.traces = s.traces.empty() ? nullptr : s.traces.data();
        return c;
    }
    static std::vector<rtm_b200_shot> to_c(const std::vector<ShotRecord>& v) {
        std::vector<rtm_b200_shot> c;
        c.reserve(v.size());
        for (const auto& s : v) c.push_back(to_c1(s));
        return c;
    }
    rtm_b200_config cfg_{};
    rtm_b200_engine* h_ = nullptr;
};

// For factory_b200.cpp: the engine for a name, or null.
std::unique_ptr<RTMEngine> make_b200_engine(const std::string& name) {
    if (name == "b200") return std::make_unique<B200RTM>(RTM_B200_MODE_PLAIN);
    if (name == "b200-batch") return std::make_unique<B200RTM>(RTM_B200_MODE_BATCH);
    if (name == "b200-serve") return std::make_unique<B200RTM>(RTM_B200_MODE_SERVE);
    return nullptr;
}

}  // namespace rtm
