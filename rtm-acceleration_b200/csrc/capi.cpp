// capi.cpp -- the extern "C" boundary of librtm_b200.so (declared in
// include/rtm_b200.h).  Every entry point catches every C++ exception and turns
// it into a status code; nothing throws across the ABI.
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <string>

#include "engine.hpp"
#include "rtm_b200.h"

struct rtm_b200_engine {
    std::unique_ptr<rtmb::Engine> e;
};

namespace {
std::mutex g_err_mu;
std::string g_create_error;

void copy_str(const std::string& s, char* buf, size_t len) {
    if (!buf || len == 0) return;
    const size_t n = s.size() < len - 1 ? s.size() : len - 1;
    std::memcpy(buf, s.data(), n);
    buf[n] = '\0';
}

template <typename F>
int guarded(rtm_b200_engine* h, F&& f) {
    if (!h || !h->e) return RTM_B200_EINVAL;
    try {
        return f(*h->e);
    } catch (const std::bad_alloc&) {
        return h->e->fail(RTM_B200_ENOMEM, "host allocation failed");
    } catch (const std::exception& ex) {
        return h->e->fail(RTM_B200_EINVAL, ex.what());
    } catch (...) {
        return h->e->fail(RTM_B200_EINVAL, "unknown error");
    }
}
}  // namespace

extern "C" {

void rtm_b200_config_init(rtm_b200_config* c) {
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    c->struct_size = (int)sizeof(*c);
    c->mode = RTM_B200_MODE_PLAIN;
    c->nb = 60;
    c->order = 8;
    c->sponge_alpha = 0.0053f;
    c->store_interval = 1;
    c->f0 = 12.0f;
    c->verbose = 0;
    c->snap_precision = RTM_B200_SNAP_F32;
    c->arithmetic = RTM_B200_ARITH_AUTO;
    c->accumulation = RTM_B200_ACC_COMPENSATED;
}

int rtm_b200_create(const rtm_b200_config* cfg, rtm_b200_engine** out) {
    if (!cfg || !out) return RTM_B200_EINVAL;
    *out = nullptr;
    if (cfg->struct_size != (int)sizeof(rtm_b200_config)) {
        std::lock_guard<std::mutex> lk(g_err_mu);
        g_create_error = "rtm_b200_config.struct_size does not match this library";
        return RTM_B200_EINVAL;
    }
    try {
        auto h = std::make_unique<rtm_b200_engine>();
        h->e = std::make_unique<rtmb::Engine>(*cfg);
        const int rc = h->e->init();
        if (rc != RTM_B200_OK) {
            std::lock_guard<std::mutex> lk(g_err_mu);
            g_create_error = h->e->last_error();
            return rc;
        }
        *out = h.release();
        return RTM_B200_OK;
    } catch (const std::exception& ex) {
        std::lock_guard<std::mutex> lk(g_err_mu);
        g_create_error = ex.what();
        return RTM_B200_ENOMEM;
    }
}

int rtm_b200_destroy(rtm_b200_engine* h) {
    if (!h) return RTM_B200_EINVAL;
    delete h;
    return RTM_B200_OK;
}

int rtm_b200_setup(rtm_b200_engine* h, const float* vel, int nx, int nz, float dx, float dz, float ox, float oz,
                   int nt, float dt) {
    return guarded(h, [&](rtmb::Engine& e) { return e.setup(vel, nx, nz, dx, dz, ox, oz, nt, dt); });
}

int rtm_b200_migrate(rtm_b200_engine* h, const rtm_b200_shot* shots, int nshots, float* image, float* illum) {
    return guarded(h, [&](rtmb::Engine& e) { return e.migrate(shots, nshots, image, illum, nullptr, nullptr); });
}

int rtm_b200_migrate_f64(rtm_b200_engine* h, const rtm_b200_shot* shots, int nshots, double* image,
                         double* illum) {
    return guarded(h, [&](rtmb::Engine& e) { return e.migrate(shots, nshots, nullptr, nullptr, image, illum); });
}

int rtm_b200_postprocess(rtm_b200_engine* h, float eps_relative, int compensate_filtered, float* illum_out,
                         float* filtered_out) {
    return guarded(h, [&](rtmb::Engine& e) {
        return e.postprocess(eps_relative, compensate_filtered != 0, illum_out, filtered_out);
    });
}

int rtm_b200_model_shots(rtm_b200_engine* h, const rtm_b200_shot* shots, int nshots, float* traces_out) {
    return guarded(h, [&](rtmb::Engine& e) { return e.model_shots(shots, nshots, traces_out); });
}

int rtm_b200_forward(rtm_b200_engine* h, const rtm_b200_shot* shot, float* snapshots, float* recorded) {
    return guarded(h, [&](rtmb::Engine& e) {
        if (!shot) return e.fail(RTM_B200_EINVAL, "null shot");
        return e.forward(shot, snapshots, recorded);
    });
}

int rtm_b200_backward(rtm_b200_engine* h, const rtm_b200_shot* shot, const float* snapshots, float* image,
                      float* illum) {
    return guarded(h, [&](rtmb::Engine& e) {
        if (!shot) return e.fail(RTM_B200_EINVAL, "null shot");
        return e.backward(shot, snapshots, image, illum);
    });
}

int rtm_b200_imaging(rtm_b200_engine* h, const float* fwd_snapshot, const float* bwd_extended, float* image,
                     float* illum) {
    return guarded(h, [&](rtmb::Engine& e) { return e.imaging(fwd_snapshot, bwd_extended, image, illum); });
}

int rtm_b200_num_snapshots(const rtm_b200_engine* h) { return (h && h->e) ? h->e->num_snapshots() : 0; }

long long rtm_b200_snapshot_bytes(const rtm_b200_engine* h) { return (h && h->e) ? h->e->snapshot_bytes() : 0; }

int rtm_b200_get_times(const rtm_b200_engine* h, rtm_b200_times* out) {
    if (!h || !h->e || !out) return RTM_B200_EINVAL;
    *out = h->e->times;
    return RTM_B200_OK;
}

int rtm_b200_reset_times(rtm_b200_engine* h) {
    if (!h || !h->e) return RTM_B200_EINVAL;
    h->e->times = rtm_b200_times{};
    return RTM_B200_OK;
}

int rtm_b200_device_name(const rtm_b200_engine* h, char* buf, size_t len) {
    if (!h || !h->e) return RTM_B200_EINVAL;
    copy_str(h->e->device_name(), buf, len);
    return RTM_B200_OK;
}

int rtm_b200_autotune_report(const rtm_b200_engine* h, char* buf, size_t len) {
    if (!h || !h->e || !buf) return RTM_B200_EINVAL;
    std::string js = "[";
    for (size_t i = 0; i < h->e->tune_log_.size(); ++i) {
        const auto& r = h->e->tune_log_[i];
        js += i ? ", {" : "{";
        js += "\"key\": [";
        for (size_t k = 0; k < r.key.size(); ++k) js += (k ? ", " : "") + std::to_string(r.key[k]);
        js += "], \"us_per_step\": [";
        for (size_t k = 0; k < r.us_per_step.size(); ++k) {
            char t[32];
            std::snprintf(t, sizeof t, "%s%.3f", k ? ", " : "", r.us_per_step[k]);
            js += t;
        }
        auto choice = [](const rtmb::Engine::TuneChoice& c) {
            return std::string("{\"kernel\": \"") + (c.kind == 1 ? "march" : "ring") + "\", \"warps\": " +
                   std::to_string(c.warps) + ", \"tile_x\": " + std::to_string(c.tile_x) + ", \"stages\": " + std::to_string(c.stages) + ", \"march_m\": " +
                   std::to_string(c.march_m) + ", \"spare\": " + std::to_string(c.spare) + "}";
        };
        js += "], \"candidates\": [";
        for (size_t k = 0; k < r.cands.size(); ++k) js += (k ? ", " : "") + choice(r.cands[k]);
        js += "], \"pick\": " + choice(r.pick) + "}";
    }
    for (const auto& t : h->e->inflight_log_) {
        js += js.size() > 1 ? ", {" : "{";
        js += "\"kind\": \"shots_in_flight\", \"key\": [";
        for (size_t k = 0; k < t.key.size(); ++k) js += (k ? ", " : "") + std::to_string(t.key[k]);
        js += "], \"candidates\": [";
        for (size_t k = 0; k < t.cands.size(); ++k) js += (k ? ", " : "") + std::to_string(t.cands[k]);
        js += "], \"shots_per_s\": [";
        for (size_t k = 0; k < t.shots_per_s.size(); ++k) {
            char v[32];
            std::snprintf(v, sizeof v, "%s%.3f", k ? ", " : "", t.shots_per_s[k]);
            js += v;
        }
        js += "], \"pick\": " + std::to_string(t.pick) + "}";
    }
    js += "]";
    copy_str(js, buf, len);
    return js.size() < len ? RTM_B200_OK : RTM_B200_EINVAL;
}

int rtm_b200_last_error(const rtm_b200_engine* h, char* buf, size_t len) {
    if (!h || !h->e) {
        std::lock_guard<std::mutex> lk(g_err_mu);
        copy_str(g_create_error, buf, len);
        return RTM_B200_OK;
    }
    copy_str(h->e->last_error(), buf, len);
    return RTM_B200_OK;
}

int rtm_b200_submit(rtm_b200_engine* h, const rtm_b200_request* req, long long* ticket) {
    return guarded(h, [&](rtmb::Engine& e) { return e.submit(req, ticket); });
}

int rtm_b200_serve_step(rtm_b200_engine* h, int max_steps, int* pending) {
    return guarded(h, [&](rtmb::Engine& e) { return e.serve_step(max_steps, pending); });
}

int rtm_b200_poll(rtm_b200_engine* h, long long ticket, rtm_b200_request_status* st, float* image, float* illum) {
    return guarded(h, [&](rtmb::Engine& e) { return e.poll(ticket, st, image, illum); });
}

int rtm_b200_drain(rtm_b200_engine* h) {
    return guarded(h, [&](rtmb::Engine& e) { return e.drain(); });
}

double rtm_b200_clock(const rtm_b200_engine* h) { return (h && h->e) ? h->e->clock() : 0.0; }

int rtm_b200_memory_probe(rtm_b200_engine* h, size_t bytes, int iters, double* gbps) {
    return guarded(h, [&](rtmb::Engine& e) { return e.memory_probe(bytes, iters, gbps); });
}

int rtm_b200_l2_probe(rtm_b200_engine* h, size_t bytes, int reps, double* gbps) {
    return guarded(h, [&](rtmb::Engine& e) { return e.l2_probe(bytes, reps, gbps); });
}

}  // extern "C"

// ---------------------------------------------------------------- host numerics
#include <algorithm>
#include <cmath>

#include "numerics.hpp"

extern "C" {

int rtm_b200_stencil_coefficients(int order, float* c) {
    if (!c) return RTM_B200_EINVAL;
    if (!rtmb::stencil_coefficients(order, c)) return RTM_B200_EINVAL;
    return order / 2;
}

float rtm_b200_max_stable_dt(float vmax, float dx, float dz, int order) {
    if (rtmb::stencil_half(order) < 0) return -1.0f;
    return rtmb::max_stable_dt(vmax, dx, dz, order);
}

float rtm_b200_ricker(float t, float f0) { return rtmb::ricker(t, f0); }

float rtm_b200_points_per_wavelength(float vmin, float f0, float dx, float dz) {
    return rtmb::points_per_wavelength(vmin, f0, dx, dz);
}

// Reference seismic_io.cpp:18-35: zero up to i0 = floor((offset/v + t_pad)/dt),
// then a raised-cosine ramp over the next max(1, t_taper/dt) samples.
void rtm_b200_mute_direct_wave(const rtm_b200_shot* s, float* traces, float v_surface, float t_pad,
                               float t_taper) {
    if (!s || !traces || v_surface <= 0.0f) return;
    for (int ir = 0; ir < s->nrec; ++ir) {
        const float ddx = s->rx[ir] - s->sx;
        const float ddz = s->rz[ir] - s->sz;
        const float off = std::sqrt(ddx * ddx + ddz * ddz);
        const float t0 = off / v_surface + t_pad;
        const int i0 = (int)(t0 / s->dt);
        const int i1 = i0 + std::max(1, (int)(t_taper / s->dt));
        float* tr = traces + (size_t)ir * s->nt;
        for (int it = 0; it < s->nt && it < i1; ++it) {
            if (it <= i0) {
                tr[it] = 0.0f;
                continue;
            }
            const float u = (float)(it - i0) / (float)(i1 - i0);
            tr[it] *= 0.5f * (1.0f - std::cos((float)M_PI * u));
        }
    }
}

}  // extern "C"
