// serve.cu -- the continuous-batching serving loop of rtmb::Engine.
//
// Requests (each with its own model, grid, order, time axis and shots) queue on
// the host.  Every serve_step() retires the shots that finished, completes
// requests whose shots are all done (their FP64 stack is extracted and copied
// to pinned host memory asynchronously; an event marks it ready), admits queued
// shots into free slots as long as the snapshot arena has room for them (the
// admission currency is snapshot bytes), then advances every shot in flight by
// a chunk of time steps.  Shots of different requests share each step launch
// (one launch per stencil order present), so work that arrives while others run
// overlaps on the device.
#include <algorithm>
#include <cstring>

#include "engine.hpp"
#include "kernels.hpp"

namespace rtmb {

int Engine::serve_init(const Model& first) {
    if (serve_ready_) return RTM_B200_OK;
    const int max_nx = cfg_.serve_max_nx > 0 ? cfg_.serve_max_nx : std::max(first.g.nx, 2000);
    const int max_nz = cfg_.serve_max_nz > 0 ? cfg_.serve_max_nz : std::max(first.g.nz, 800);
    const GridDims gmax = make_grid(max_nx, max_nz, cfg_.nb, kMaxHalf);
    const int nslots = cfg_.max_shots_in_flight > 0 ? cfg_.max_shots_in_flight : 32;
    RTMB_TRY(ensure_pool(nslots, gmax.nxe, gmax.ldz));
    size_t freeb = 0, totalb = 0;
    RTMB_CUDA(cudaMemGetInfo(&freeb, &totalb));
    // Leave room for per-slot tables, request tables and images.
    const size_t per_slot_aux = (size_t)gmax.nx * gmax.lds * 16 + (size_t)gmax.nx * 6000 * 4;
    size_t budget = cfg_.device_mem_budget > 0 ? (size_t)cfg_.device_mem_budget : (size_t)(0.85 * (double)freeb);
    const size_t reserve = (size_t)nslots * per_slot_aux + ((size_t)2 << 30);
    size_t arena = budget > reserve ? budget - reserve : 0;
    arena = std::min(arena, freeb > reserve ? freeb - reserve : 0);
    arena_.release();
    if (arena && arena_.alloc(arena) != cudaSuccess) {
        cudaGetLastError();
        return fail(RTM_B200_ENOMEM, "cannot allocate the serving snapshot arena");
    }
    alloc_.reset(arena_.bytes());
    serve_ready_ = true;
    return RTM_B200_OK;
}

int Engine::submit(const rtm_b200_request* req, long long* ticket) {
    if (!inited_) return fail(RTM_B200_ESTATE, "engine not initialised");
    if (cfg_.mode != RTM_B200_MODE_SERVE) return fail(RTM_B200_ESTATE, "submit needs the serving engine");
    if (!req || !ticket) return fail(RTM_B200_EINVAL, "null request");
    RTMB_CUDA(cudaSetDevice(device_));
    auto m = std::make_unique<Model>();
    int rc = build_model(*m, req->vel, req->nx, req->nz, req->dx, req->dz, req->ox, req->oz, req->order, req->nt,
                         req->dt, req->store_interval, req->f0);
    if (rc != RTM_B200_OK) return RTM_B200_EREJECTED;
    // CFL (reference src/main.cpp:190-192): an unstable request is rejected.
    const float dt_max = max_stable_dt(m->vmax, m->dx, m->dz, m->order);
    if (req->dt > dt_max) return fail(RTM_B200_EREJECTED, "request violates the CFL condition");
    rc = copy_shots(*m, req->shots, req->nshots, true);
    if (rc != RTM_B200_OK) return RTM_B200_EREJECTED;
    if (req->nshots <= 0) return fail(RTM_B200_EREJECTED, "request has no shots");
    RTMB_TRY(serve_init(*m));
    if (m->g.nxe > nxe_cap_ || m->g.ldz > ldz_cap_)
        return fail(RTM_B200_EREJECTED, "request grid exceeds the serving pool");
    const size_t need = snap_alloc_bytes(*m, m->g);
    if (need > alloc_.capacity()) return fail(RTM_B200_EREJECTED, "one shot's snapshots exceed the device budget");
    const size_t n = (size_t)m->g.nx * m->g.lds;
    RTMB_CUDA(m->img64.alloc(n * 8));
    RTMB_CUDA(m->ill64.alloc(n * 8));
    RTMB_CUDA(cudaMemsetAsync(m->img64.get(), 0, n * 8, stream_));
    RTMB_CUDA(cudaMemsetAsync(m->ill64.get(), 0, n * 8, stream_));
    m->id = next_ticket_++;
    m->t_submit = clock();
    m->state = 0;
    for (int i = 0; i < req->nshots; ++i) serve_q_.emplace_back(m.get(), i);
    *ticket = m->id;
    requests_[m->id] = std::move(m);
    return RTM_B200_OK;
}

// Requests whose shots have all retired: enqueue the extraction of their image
// and the copy to pinned host memory, to be collected when the event fires.
int Engine::serve_finish_models() {
    for (auto& kv : requests_) {
        Model& m = *kv.second;
        if (m.state != 1 || m.shots_done < (int)m.shots.size()) continue;
        auto f = std::make_unique<Finishing>();
        f->ticket = kv.first;
        const size_t n = (size_t)m.g.nx * m.g.nz;
        if (f->host.reserve(2 * n * 4) != cudaSuccess) {
            cudaGetLastError();
            return fail(RTM_B200_ENOMEM, "pinned result buffer");
        }
        // dense FP32 output staged in the request's (unused) running-image buffer
        RTMB_CUDA(m.img.reserve(2 * n * 4));
        float* dense = m.img.get<float>();
        const int row0 = m.g.nb - m.g.zs0;
        RTMB_CUDA(launch_extract_f64_to_f32(m.img64.get<double>(), m.g.lds, row0, dense, m.g.nx, m.g.nz, stream_));
        RTMB_CUDA(launch_extract_f64_to_f32(m.ill64.get<double>(), m.g.lds, row0, dense + n, m.g.nx, m.g.nz, stream_));
        RTMB_CUDA(cudaMemcpyAsync(f->host.get(), dense, 2 * n * 4, cudaMemcpyDeviceToHost, stream_));
        RTMB_CUDA(cudaEventCreateWithFlags(&f->ev, cudaEventDisableTiming));
        RTMB_CUDA(cudaEventRecord(f->ev, stream_));
        launches_ += 2;
        m.state = 3;   // finishing
        finishing_.push_back(std::move(f));
    }
    return RTM_B200_OK;
}

int Engine::serve_collect(bool wait) {
    for (size_t i = 0; i < finishing_.size();) {
        Finishing& f = *finishing_[i];
        cudaError_t q = wait ? cudaEventSynchronize(f.ev) : cudaEventQuery(f.ev);
        if (q == cudaErrorNotReady) { ++i; continue; }
        RTMB_CUDA(q);
        Model& m = *requests_[f.ticket];
        const size_t n = (size_t)m.g.nx * m.g.nz;
        m.out_img.assign(f.host.get<float>(), f.host.get<float>() + n);
        m.out_ill.assign(f.host.get<float>() + n, f.host.get<float>() + 2 * n);
        m.t_finish = clock();
        m.state = 2;
        // release the request's device tables
        m.vdt2.release(); m.wavelet.release(); m.wz.release();
        m.img.release(); m.ill.release(); m.img64.release(); m.ill64.release();
        cudaEventDestroy(f.ev);
        finishing_.erase(finishing_.begin() + (long)i);
    }
    return RTM_B200_OK;
}

int Engine::serve_admit() {
    int admitted = 0;
    // FIFO over shots; admit_from stops at the first shot that does not fit.
    RTMB_TRY(admit_from(serve_q_, false, nullptr, nullptr, &admitted));
    for (auto& j : jobs_)
        if (j.active && j.m->state == 0) j.m->state = 1;
    return RTM_B200_OK;
}

int Engine::serve_step(int max_steps, int* pending) {
    if (cfg_.mode != RTM_B200_MODE_SERVE) return fail(RTM_B200_ESTATE, "serve_step needs the serving engine");
    RTMB_CUDA(cudaSetDevice(device_));
    int budget = max_steps > 0 ? max_steps : 1;
    while (true) {
        RTMB_TRY(serve_collect(false));
        RTMB_TRY(retire_finished());
        RTMB_TRY(serve_finish_models());
        RTMB_TRY(serve_admit());
        if (active_jobs() == 0 || budget <= 0) break;
        int remaining = 0;
        for (const auto& j : jobs_)
            if (j.active) remaining = std::max(remaining, (int)(j.total - (g_ - j.g0)));
        const int c = std::min({cfg_.chunk_steps > 0 ? cfg_.chunk_steps : 64, remaining, budget});
        RTMB_TRY(run_chunk(c));
        times.kernel_launches = launches_;
        budget -= c;
    }
    int p = 0;
    for (auto& kv : requests_) p += kv.second->state != 2 ? 1 : 0;
    if (pending) *pending = p;
    return RTM_B200_OK;
}

int Engine::drain() {
    int pending = 1;
    while (pending > 0) {
        RTMB_TRY(serve_step(1 << 30, &pending));
        if (pending > 0 && active_jobs() == 0) {
            if (!serve_q_.empty()) return fail(RTM_B200_ENOMEM, "queued shots can never be admitted");
            RTMB_TRY(serve_collect(true));
            int p = 0;
            for (auto& kv : requests_) p += kv.second->state != 2 ? 1 : 0;
            pending = p;
        }
    }
    return check_device_error();
}

int Engine::poll(long long ticket, rtm_b200_request_status* st, float* img, float* ill) {
    auto it = requests_.find(ticket);
    if (it == requests_.end()) return fail(RTM_B200_ENOTFOUND, "unknown ticket");
    RTMB_TRY(serve_collect(false));
    Model& m = *it->second;
    if (st) {
        st->state = m.state == 3 ? 1 : m.state;
        st->shots_done = m.shots_done;
        st->submit_time = m.t_submit;
        st->start_time = m.t_start;
        st->finish_time = m.t_finish;
        st->snapshot_bytes = (double)snap_alloc_bytes(m, m.g);
    }
    if (m.state == 2) {
        if (img) std::memcpy(img, m.out_img.data(), m.out_img.size() * 4);
        if (ill) std::memcpy(ill, m.out_ill.data(), m.out_ill.size() * 4);
    }
    return RTM_B200_OK;
}

}  // namespace rtmb
