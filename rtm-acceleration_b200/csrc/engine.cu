// engine.cu -- implementation of rtmb::Engine (see engine.hpp).
#include <cudaTypedefs.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "engine.hpp"
#include "kernels.hpp"

namespace rtmb {

namespace {

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

size_t round256(size_t b) { return (b + 255) & ~(size_t)255; }

// True when p is device memory (the caller passed resident inputs/outputs).
bool is_device_ptr(const void* p) {
    if (!p) return false;
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// True when p is page-locked host memory registered with CUDA (DMA-able as is).
bool is_pinned_ptr(const void* p) {
    if (!p) return false;
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

}  // namespace

Engine::Engine(const rtm_b200_config& cfg) : cfg_(cfg) {
    // AUTO: the plain engine keeps the reference's unfused IEEE arithmetic (bit
    // for bit); batch and serve, whose per-shot sums are compensated and whose
    // gate is a tolerance against FP64, use fused multiply-adds.
    // Modelling (the synthetic-data generator) always runs IEEE under AUTO, so
    // that its shot files are the reference's byte for byte.
    auto_arith_ = cfg_.arithmetic == RTM_B200_ARITH_AUTO;
    if (auto_arith_)
        cfg_.arithmetic = cfg_.mode == RTM_B200_MODE_PLAIN ? RTM_B200_ARITH_IEEE : RTM_B200_ARITH_FMA;
    f64_ = cfg_.arithmetic == RTM_B200_ARITH_FP64;
    t0_ = std::chrono::steady_clock::now();
}

Engine::~Engine() {
    if (inited_) {
        cudaSetDevice(device_);
        cudaStreamSynchronize(stream_);
        if (graph_) cudaGraphExecDestroy(graph_);
        if (copy_stream_) cudaStreamSynchronize(copy_stream_);
        for (auto& s : slots_) {
            if (s.staged) cudaEventDestroy(s.staged);
            if (s.free_ev) cudaEventDestroy(s.free_ev);
            if (s.tr_ready) cudaEventDestroy(s.tr_ready);
        }
        if (ev0_) cudaEventDestroy(ev0_);
        if (ev1_) cudaEventDestroy(ev1_);
        if (tune_ev0_) cudaEventDestroy(tune_ev0_);
        if (tune_ev1_) cudaEventDestroy(tune_ev1_);
        for (auto& e : chunk_ev_)
            if (e) cudaEventDestroy(e);
        for (auto& f : finishing_)
            if (f && f->ev) cudaEventDestroy(f->ev);
        if (copy_stream_) cudaStreamDestroy(copy_stream_);
        if (stream_) cudaStreamDestroy(stream_);
    }
}

double Engine::clock() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count();
}

int Engine::init() {
    if (cfg_.mode < RTM_B200_MODE_PLAIN || cfg_.mode > RTM_B200_MODE_SERVE)
        return fail(RTM_B200_EINVAL, "unknown engine mode");
    if (cfg_.arithmetic < RTM_B200_ARITH_IEEE || cfg_.arithmetic > RTM_B200_ARITH_FP64)
        return fail(RTM_B200_EINVAL, "unknown arithmetic");
    if (cfg_.snap_precision < RTM_B200_SNAP_F32 || cfg_.snap_precision > RTM_B200_SNAP_RECON)
        return fail(RTM_B200_EINVAL, "unknown snapshot precision");
    if (f64_ && cfg_.snap_precision != RTM_B200_SNAP_F32)
        return fail(RTM_B200_EINVAL, "the FP64 engine stores FP64 snapshots (snap_precision must be F32)");
    if (cfg_.snap_precision == RTM_B200_SNAP_RECON && cfg_.mode == RTM_B200_MODE_PLAIN)
        return fail(RTM_B200_EINVAL, "source reconstruction needs the batch or serve engine (the plain engine keeps "
                                     "the reference's snapshots, bit for bit)");
    recon_ = cfg_.snap_precision == RTM_B200_SNAP_RECON;
    nbuf_ = recon_ ? kReconBuffers : kFieldBuffers;
    if (cfg_.tile_cols != 0 && cfg_.tile_cols != 16 && cfg_.tile_cols != 32)
        return fail(RTM_B200_EINVAL, "tile_cols must be 0, 16 or 32");
    int n = 0;
    RTMB_CUDA(cudaGetDeviceCount(&n));
    if (cfg_.device < 0 || cfg_.device >= n) return fail(RTM_B200_ECUDA, "CUDA device ordinal out of range");
    device_ = cfg_.device;
    RTMB_CUDA(cudaSetDevice(device_));
    cudaDeviceProp prop{};
    RTMB_CUDA(cudaGetDeviceProperties(&prop, device_));
    if (prop.major != 10)
        return fail(RTM_B200_ECUDA, std::string("librtm_b200 is built for sm_100a (B200); device is ") + prop.name);
    device_name_ = prop.name;
    if (!tensor_map_encoder()) return fail(RTM_B200_ECUDA, "cuTensorMapEncodeTiled is unavailable");
    RTMB_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    RTMB_CUDA(cudaStreamCreateWithFlags(&copy_stream_, cudaStreamNonBlocking));
    RTMB_CUDA(cudaEventCreate(&ev0_));
    RTMB_CUDA(cudaEventCreate(&ev1_));
    for (auto& e : chunk_ev_) RTMB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    RTMB_CUDA(counter_.alloc(sizeof(long long)));
    RTMB_CUDA(errword_.alloc(sizeof(int)));
    RTMB_CUDA(cudaMemsetAsync(counter_.get(), 0, sizeof(long long), stream_));
    RTMB_CUDA(cudaMemsetAsync(errword_.get(), 0, sizeof(int), stream_));
    RTMB_CUDA(cudaStreamSynchronize(stream_));
    tile_x_ = cfg_.tile_cols == 32 ? 32 : 16;
    warps_ = tile_x_ == 32 ? 8 : 4;
    // Test hook: RTM_B200_RING_WARPS=8 with tile_cols 16 pins the 8-warp x
    // 16-column shape (its per-column path), so tests can compare it with the
    // column-pair shapes.
    if (const char* w = std::getenv("RTM_B200_RING_WARPS"))
        if (tile_x_ == 16 && cfg_.tile_cols != 0 && std::atoi(w) == 8) warps_ = 8;
    // Test hook: RTM_B200_BAND_SHIFT=0 keeps every job's bands at row 0 and tile
    // columns at column 0, so tests can compare shifted and unshifted tilings
    // bit for bit.
    if (const char* b = std::getenv("RTM_B200_BAND_SHIFT")) band_shift_ = std::atoi(b) != 0;
    autotune_ = cfg_.tile_cols == 0;
    // Failure-detection test hook: the first step launch leaves this tile's
    // stage empty, so the kernel's bounded wait must give up and report.
    if (const char* st = std::getenv("RTM_B200_STALL_TILE")) stall_tile_ = std::atoi(st);
    // RTM_B200_STEP_KERNEL=ring|march pins the step kernel (the autotuner then
    // only tunes that kernel's parameters); tests use it to check both kernels.
    pin_kind_ = -1;
    if (const char* k = std::getenv("RTM_B200_STEP_KERNEL")) {
        if (!std::strcmp(k, "ring")) pin_kind_ = kStepRing;
        if (!std::strcmp(k, "march")) pin_kind_ = kStepMarch;
    }
    if (stall_tile_ >= 0) pin_kind_ = kStepRing;   // the hook needs the ring kernel's waits
    if (pin_kind_ >= 0) kind_ = pin_kind_;
    RTMB_CUDA(cudaEventCreate(&tune_ev0_));
    RTMB_CUDA(cudaEventCreate(&tune_ev1_));
    inited_ = true;
    return RTM_B200_OK;
}

// ------------------------------------------------------------------ set-up
int Engine::validate_params(int nx, int nz, float dx, float dz, int order, int nb, int si, int nt, float dt,
                            float f0, const float* vel, float* vmin, float* vmax) {
    const int half = stencil_half(order);
    if (half < 0) return fail(RTM_B200_EINVAL, "unsupported spatial order (use 2, 4, 6, 8, 10 or 12)");
    if (nb < half + 1) return fail(RTM_B200_EINVAL, "--nb must be at least order/2 + 1");
    if (si < 1) return fail(RTM_B200_EINVAL, "--store-interval must be >= 1");
    if (nx <= 0 || nz <= 0) return fail(RTM_B200_EINVAL, "velocity nx/nz must be positive");
    if (nt <= 0) return fail(RTM_B200_EINVAL, "nt must be positive");
    if (!(dt > 0.0f) || !(dx > 0.0f) || !(dz > 0.0f) || !(f0 > 0.0f))
        return fail(RTM_B200_EINVAL, "dt, dx, dz and f0 must be positive");
    if (!vel) return fail(RTM_B200_EINVAL, "velocity model is null");
    float lo = vel[0], hi = vel[0];
    const size_t n = (size_t)nx * nz;
    for (size_t i = 0; i < n; ++i) {
        const float v = vel[i];
        if (!(v > 0.0f) || v > 20000.0f) return fail(RTM_B200_EINVAL, "velocity model contains a non-physical value");
        lo = std::min(lo, v);
        hi = std::max(hi, v);
    }
    *vmin = lo;
    *vmax = hi;
    return RTM_B200_OK;
}

int Engine::build_model(Model& m, const float* vel, int nx, int nz, float dx, float dz, float ox, float oz,
                        int order, int nt, float dt, int si, float f0) {
    RTMB_TRY(validate_params(nx, nz, dx, dz, order, cfg_.nb, si, nt, dt, f0, vel, &m.vmin, &m.vmax));
    m.half = stencil_half(order);
    m.order = order;
    m.g = make_grid(nx, nz, cfg_.nb, m.half);
    m.dx = dx; m.dz = dz; m.ox = ox; m.oz = oz;
    m.nt = nt; m.dt = dt; m.si = si; m.f0 = f0; m.alpha = cfg_.sponge_alpha;
    m.nsnap = (nt - 1) / si + 1;
    m.coef = scaled_coefficients(order, dx, dz);

    const GridDims& g = m.g;
    // (v dt)^2 per model column, extended in depth by replicating the top and
    // bottom rows (reference rtm_cpu.cpp:33-42); x is extended in-kernel.
    std::vector<float> t((size_t)nx * g.ldz, 0.0f);
    const float dt2 = dt * dt;
    for (int ix = 0; ix < nx; ++ix)
        for (int ize = 0; ize < g.nze; ++ize) {
            const int iz = std::min(std::max(ize - g.nb, 0), nz - 1);
            const float v = vel[(size_t)ix * nz + iz];
            t[(size_t)ix * g.ldz + ize] = v * v * dt2;
        }
    RTMB_CUDA(m.vdt2.alloc(t.size() * sizeof(float)));
    RTMB_CUDA(cudaMemcpy(m.vdt2.get(), t.data(), t.size() * sizeof(float), cudaMemcpyHostToDevice));
    const std::vector<float> w = ricker_wavelet(nt, dt, f0);
    RTMB_CUDA(m.wavelet.alloc(w.size() * sizeof(float)));
    RTMB_CUDA(cudaMemcpy(m.wavelet.get(), w.data(), w.size() * sizeof(float), cudaMemcpyHostToDevice));
    std::vector<float> wz((size_t)g.ldz, 0.0f);
    for (int i = 0; i < g.nze; ++i) wz[(size_t)i] = cerjan_taper(i, g.nze, g.nb, m.alpha);
    RTMB_CUDA(m.wz.alloc(wz.size() * sizeof(float)));
    RTMB_CUDA(cudaMemcpy(m.wz.get(), wz.data(), wz.size() * sizeof(float), cudaMemcpyHostToDevice));
    return RTM_B200_OK;
}

int Engine::setup(const float* vel, int nx, int nz, float dx, float dz, float ox, float oz, int nt, float dt) {
    if (!inited_) return fail(RTM_B200_ESTATE, "engine not initialised");
    if (active_jobs()) return fail(RTM_B200_ESTATE, "setup while shots are in flight");
    RTMB_CUDA(cudaSetDevice(device_));
    auto m = std::make_unique<Model>();
    RTMB_TRY(build_model(*m, vel, nx, nz, dx, dz, ox, oz, cfg_.order, nt, dt, cfg_.store_interval, cfg_.f0));
    model_ = std::move(m);
    keep_snap_ = false;
    stack_ready_ = false;
    return RTM_B200_OK;
}

int Engine::snap_type() const {
    if (f64_) return kSnapF64;
    switch (cfg_.snap_precision) {
        case RTM_B200_SNAP_RECON: return kSnapNone;
        case RTM_B200_SNAP_BF16: return kSnapBF16;
        case RTM_B200_SNAP_F16: return kSnapF16;
        default: return kSnapF32;
    }
}

size_t Engine::snap_alloc_bytes(const Model& m, const GridDims& gs) const {
    const int st = snap_type();
    if (st == kSnapNone)   // boundary strips of levels 1..nt-1
        return round256((size_t)std::max(m.nt - 1, 1) * strip_cells(gs.nx, gs.nz, m.half) * 4);
    const size_t es = st == kSnapF64 ? 8 : (st == kSnapF32 ? 4 : 2);
    size_t b = round256((size_t)m.nsnap * gs.nx * gs.lds * es);
    if (st == kSnapBF16 || st == kSnapF16) b += round256((size_t)m.nsnap * gs.nx * gs.ntz);
    return b;
}

long long Engine::snapshot_bytes() const {
    if (!model_) return 0;
    return (long long)snap_alloc_bytes(*model_, model_->g);
}

int Engine::copy_shots(Model& m, const rtm_b200_shot* shots, int nshots, bool need_traces) {
    if (nshots < 0 || (nshots > 0 && !shots)) return fail(RTM_B200_EINVAL, "shots array is null");
    m.shots.clear();
    m.shots.reserve((size_t)nshots);
    for (int i = 0; i < nshots; ++i) {
        const rtm_b200_shot& s = shots[i];
        ShotData d;
        d.sx = s.sx; d.sz = s.sz; d.nrec = s.nrec; d.nt = s.nt; d.dt = s.dt;
        if (s.nrec < 0 || (s.nrec > 0 && (!s.rx || !s.rz))) return fail(RTM_B200_EINVAL, "receiver arrays are null");
        if (need_traces) {
            if (s.nrec > 0 && !s.traces) return fail(RTM_B200_EINVAL, "shot traces are null");
            if (s.nt < m.nt) return fail(RTM_B200_EINVAL, "shot has fewer samples than the time axis");
        }
        d.rx.assign(s.rx, s.rx + s.nrec);
        d.rz.assign(s.rz, s.rz + s.nrec);
        d.traces = s.traces;
        if (s.window_nx == 0 && s.window_x0 == 0) {
            d.x0 = 0;
            d.wnx = m.g.nx;
        } else {
            if (s.window_x0 < 0 || s.window_nx < 1 || s.window_x0 + s.window_nx > m.g.nx)
                return fail(RTM_B200_EINVAL, "aperture window outside the model");
            d.x0 = s.window_x0;
            d.wnx = s.window_nx;
        }
        m.shots.push_back(std::move(d));
    }
    m.next_shot = 0;
    m.shots_done = 0;
    return RTM_B200_OK;
}

// -------------------------------------------------------------- pool, slots
StepVariant Engine::variant(int half) const {
    StepVariant v;
    v.f64 = f64_;
    v.half = half;
    v.tile_x = tile_x_;
    v.warps = f64_ ? 8 : warps_;
    v.spare = spare_ != 0 && step_ctas_per_sm(v) > 1;
    v.exact = exact();
    // the march kernel has no reconstruction, nor shifted bands
    v.kind = (f64_ || recon_ || shifted_bands()) ? kStepRing : kind_;
    v.march_m = march_m_;
    v.nstage = step_default_stages(v);
    if (stage_override_ > 0) {
        StepVariant t = v;
        t.nstage = stage_override_;
        if (step_variant_supported(t)) v.nstage = stage_override_;
    }
    return v;
}

int Engine::encode_map(int half, bool with_halo, CUtensorMap* out) {
    const StepVariant v = variant(half);
    const cuuint64_t dims[3] = {(cuuint64_t)ldz_cap_, (cuuint64_t)nxe_cap_, (cuuint64_t)pool_buffers()};
    const cuuint64_t strides[2] = {(cuuint64_t)ldz_cap_ * elem(), (cuuint64_t)ldz_cap_ * nxe_cap_ * elem()};
    const cuuint32_t box[3] = {(cuuint32_t)(with_halo ? step_box_z(v) : kTileZ),
                               (cuuint32_t)(with_halo ? step_box_x(v) : step_tile_x(v)), 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = tensor_map_encoder()(
        out, f64_ ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, pool_.get(), dims, strides,
        box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(RTM_B200_ECUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
    return RTM_B200_OK;
}

int Engine::ensure_pool(int nslots, int nxe_cap, int ldz_cap) {
    if (pool_.get() && nslots <= nslots_ && nxe_cap <= nxe_cap_ && ldz_cap == ldz_cap_) return RTM_B200_OK;
    if (active_jobs()) return fail(RTM_B200_ESTATE, "field pool resize while shots are in flight");
    RTMB_CUDA(cudaStreamSynchronize(stream_));
    if (graph_) { cudaGraphExecDestroy(graph_); graph_ = nullptr; }
    graph_sig_.clear();
    pool_.release();
    nslots_ = std::max(nslots, nslots_);
    nxe_cap_ = std::max(nxe_cap, nxe_cap_);
    ldz_cap_ = ldz_cap;
    shared_vd_uid_ = 0;
    const size_t bytes = (size_t)pool_buffers() * nxe_cap_ * ldz_cap_ * elem();
    cudaError_t e = pool_.alloc(bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(RTM_B200_ENOMEM, "cannot allocate the field pool (" + std::to_string(bytes >> 20) + " MiB)");
    }
    maps_.clear();
    slots_.resize((size_t)nslots_);
    jobs_.resize((size_t)nslots_);
    host_descs_.assign((size_t)nslots_, ShotDesc{});
    RTMB_CUDA(descs_.alloc(sizeof(ShotDesc) * nslots_));
    RTMB_CUDA(cudaMemset(descs_.get(), 0, sizeof(ShotDesc) * nslots_));
    tiles_dirty_ = true;
    return RTM_B200_OK;
}

// Loads m's (v dt)^2 table into the pool's shared buffer (zero rows below the
// table, as in a slot's copy), unless the buffer holds it already or an active
// job of another model still reads it; in that case m's shots keep loading their
// slot's copies.  Stream-ordered after every launch that read the old table.
int Engine::share_model_vdt2(const Model* m) {
    if (f64_ || shared_vd_uid_ == m->uid || m->g.nx > nxe_cap_ || m->g.ldz > ldz_cap_) return RTM_B200_OK;
    for (const auto& j : jobs_)
        if (j.active && j.m->uid == shared_vd_uid_) return RTM_B200_OK;
    const size_t buf = (size_t)nxe_cap_ * ldz_cap_ * elem();
    char* dst = pool_.get<char>() + (size_t)shared_vd_buf() * buf;
    RTMB_CUDA(cudaMemsetAsync(dst, 0, buf, stream_));
    RTMB_CUDA(cudaMemcpy2DAsync(dst, (size_t)ldz_cap_ * sizeof(float), m->vdt2.get<float>(),
                                (size_t)m->g.ldz * sizeof(float), (size_t)m->g.ldz * sizeof(float), (size_t)m->g.nx,
                                cudaMemcpyDeviceToDevice, stream_));
    shared_vd_uid_ = m->uid;
    tiles_dirty_ = true;
    return RTM_B200_OK;
}

// The largest receiver count and time axis over a model's shots.  Slots are
// sized for them (and for the full model width), so that shots of other
// aperture widths reuse the buffers: growing one would cost a device-wide
// synchronisation (cudaFree / cudaFreeHost) between two chunks of steps.
static void shot_caps(const Model& m, const ShotData& sh, size_t* nrec, int* nt) {
    *nrec = (size_t)std::max(sh.nrec, 1);
    *nt = std::max(sh.nt, m.nt);
    for (const auto& o : m.shots) {
        *nrec = std::max(*nrec, (size_t)o.nrec);
        *nt = std::max(*nt, o.nt);
    }
}

int Engine::ensure_slot(int s, const Model& m, const ShotData& sh, const GridDims& gs, bool modelling) {
    Slot& sl = slots_[(size_t)s];
    if (!sl.staged) RTMB_CUDA(cudaEventCreateWithFlags(&sl.staged, cudaEventDisableTiming));
    if (!sl.free_ev) RTMB_CUDA(cudaEventCreateWithFlags(&sl.free_ev, cudaEventDisableTiming));
    if (!sl.tr_ready) RTMB_CUDA(cudaEventCreateWithFlags(&sl.tr_ready, cudaEventDisableTiming));
    size_t nrec = 0;
    int nt = 0;
    shot_caps(m, sh, &nrec, &nt);
    const int nxe = std::max(gs.nxe, m.g.nxe);
    RTMB_CUDA(sl.wx.reserve(sizeof(float) * nxe));
    RTMB_CUDA(sl.col_start.reserve(sizeof(int) * (nxe + 1)));
    RTMB_CUDA(sl.pts.reserve(sizeof(PointEntry) * nrec));
    RTMB_CUDA(sl.ir.reserve(sizeof(int) * nrec));
    RTMB_CUDA(sl.rec_col.reserve(sizeof(int) * (nxe + 1)));
    RTMB_CUDA(sl.rec_z.reserve(sizeof(int) * nrec));
    if (!modelling) RTMB_CUDA(sl.traces.reserve(sizeof(float) * nrec * nt));
    if (modelling) RTMB_CUDA(sl.rec.reserve(sizeof(float) * nrec * m.nt));
    if (cfg_.mode != RTM_B200_MODE_PLAIN && !modelling) {
        const size_t n = std::max((size_t)gs.nx * gs.lds, (size_t)m.g.nx * m.g.lds);
        RTMB_CUDA(sl.acc.reserve(f64_ ? 2 * n * 8 : 2 * n * 4 + 2 * n * 2));
    }
    return RTM_B200_OK;
}

// --------------------------------------------------------------- scheduling
bool Engine::shifted_bands() const {
    for (const auto& j : jobs_)
        if (j.active && j.gs.z0 > 0) return true;
    return false;
}

int Engine::active_jobs() const {
    int n = 0;
    for (const auto& j : jobs_) n += j.active ? 1 : 0;
    return n;
}

int Engine::start_job(int s, Model* m, int shot, bool modelling, float* rec_host, int backward_only,
                      size_t snap_off, size_t snap_bytes, bool owns_snap) {
    const ShotData& sh = m->shots[(size_t)shot];
    Job& job = jobs_[(size_t)s];
    job = Job{};
    job.m = m;
    job.shot = shot;
    job.gs = make_grid(sh.wnx, m->g.nz, m->g.nb, m->half);
    // Band origin.  The live rows are [H, nze - H); the rows outside stay zero
    // (the reference's ring).  For the ring kernel's FMA migration jobs the
    // 128-row bands start at s, the largest multiple of 4 not above H, when
    // that covers the live rows with one band fewer: nze = 520 at order 8
    // becomes four bands of rows 4-515 instead of five, the fifth holding 8
    // rows, whose tiles cost nearly as much as full ones.  Sources and
    // receivers sit at rows >= nb >= s.  The rows outside the bands are
    // cleared once when the slot is set up and never written.
    {
        const int H = m->half, s0 = H & ~3;
        const int ntz_s = (job.gs.nze - H - s0 + kTileZ - 1) / kTileZ;
        const bool shiftable = band_shift_ && !modelling && !recon_ && !exact();
        if (shiftable && s0 > 0 && job.gs.nb >= s0 && ntz_s < job.gs.ntz) {
            job.gs.z0 = s0;
            job.gs.ntz = ntz_s;
        }
        // Columns likewise: the tile columns may start at column H (the column
        // coordinate of a TMA box has no alignment rule), which saves a tile
        // column whenever the live columns [H, nxe - H) fit in one fewer.
        job.shift_cols = shiftable && job.gs.nb >= H;
    }
    job.x0 = sh.x0;
    job.modelling = modelling;
    job.rec_host = rec_host;
    job.snap_off = snap_off;
    job.snap_bytes = snap_bytes;
    job.owns_snap = owns_snap;
    const GridDims& gs = job.gs;

    const float ox_w = m->ox + (float)sh.x0 * m->dx;
    ShotGeometry geo = build_geometry(sh.sx, sh.sz, sh.nrec, sh.rx.data(), sh.rz.data(), gs.nx, gs.nz, m->dx, m->dz,
                                      ox_w, m->oz, gs.nb);
    if (geo.nclamped > 0 && cfg_.verbose)
        std::fprintf(stderr,
                     "WARNING: %d of %d source/receiver positions fell outside the %.1f x %.1f m model and were "
                     "clamped to the edge.\n",
                     geo.nclamped, sh.nrec + 1, (gs.nx - 1) * m->dx, (gs.nz - 1) * m->dz);
    RTMB_TRY(ensure_slot(s, *m, sh, gs, modelling));
    Slot& sl = slots_[(size_t)s];
    // Receiver cells (the tile list marks the tiles that hold any).
    for (int x = 0; x < gs.nxe; ++x)
        for (int j = geo.col_start[(size_t)x]; j < geo.col_start[(size_t)x + 1]; ++j)
            job.rec_cells.emplace_back(x, geo.pts[(size_t)j].z);

    // Stage everything this job uploads in the slot's pinned buffer.
    std::vector<float> wx((size_t)gs.nxe);
    for (int i = 0; i < gs.nxe; ++i) wx[(size_t)i] = cerjan_taper(i, gs.nxe, gs.nb, m->alpha);
    const bool dev_traces = !modelling && is_device_ptr(sh.traces);
    const bool pinned_traces = !modelling && !dev_traces && is_pinned_ptr(sh.traces);
    const size_t trace_h2d = (modelling || dev_traces) ? 0 : (size_t)sh.nrec * sh.nt;   // floats uploaded
    const size_t trace_elems = pinned_traces ? 0 : trace_h2d;                           // floats staged
    size_t off = 0;
    auto take = [&](size_t bytes) { const size_t o = off; off += round256(bytes); return o; };
    const size_t o_wx = take(wx.size() * 4);
    const size_t o_cs = take(geo.col_start.size() * 4);
    const size_t o_pts = take(geo.pts.size() * sizeof(PointEntry));
    const size_t o_ir = take(geo.ir.size() * 4);
    const size_t o_rc = take(geo.rec_col.size() * 4);
    const size_t o_rz = take(geo.rec_z.size() * 4);
    const size_t o_desc = take(sizeof(ShotDesc));
    const size_t o_tr = take(trace_elems * 4);
    RTMB_CUDA(cudaEventSynchronize(sl.staged));   // previous upload from this buffer is done
    // the same layout for the largest shot of the model (see shot_caps)
    size_t cap = 0;
    {
        size_t nrec_max = 0;
        int nt_max = 0;
        shot_caps(*m, sh, &nrec_max, &nt_max);
        const size_t nxe_max = (size_t)std::max(gs.nxe, m->g.nxe);
        for (size_t b : {nxe_max * 4, (nxe_max + 1) * 4, nrec_max * sizeof(PointEntry), nrec_max * 4,
                         (nxe_max + 1) * 4, nrec_max * 4, sizeof(ShotDesc),
                         trace_elems ? nrec_max * (size_t)nt_max * 4 : (size_t)0})
            cap += round256(b);
    }
    if (cudaSuccess != sl.stage.reserve(std::max(off, cap))) {
        cudaGetLastError();
        return fail(RTM_B200_ENOMEM, "cannot allocate pinned staging memory");
    }
    char* st = sl.stage.get<char>();
    std::memcpy(st + o_wx, wx.data(), wx.size() * 4);
    std::memcpy(st + o_cs, geo.col_start.data(), geo.col_start.size() * 4);
    if (!geo.pts.empty()) std::memcpy(st + o_pts, geo.pts.data(), geo.pts.size() * sizeof(PointEntry));
    if (!geo.ir.empty()) std::memcpy(st + o_ir, geo.ir.data(), geo.ir.size() * 4);
    std::memcpy(st + o_rc, geo.rec_col.data(), geo.rec_col.size() * 4);
    if (!geo.rec_z.empty()) std::memcpy(st + o_rz, geo.rec_z.data(), geo.rec_z.size() * 4);
    if (trace_elems) std::memcpy(st + o_tr, sh.traces, trace_elems * 4);

    // Descriptor.
    ShotDesc d{};
    d.nxe = gs.nxe; d.nze = gs.nze; d.nx = gs.nx; d.nz = gs.nz; d.nb = gs.nb;
    d.model_x0 = sh.x0; d.win_nx = gs.nx;
    d.zs0 = gs.zs0; d.lds = gs.lds; d.ntz = gs.ntz;
    d.bsize = recon_ ? strip_cells(gs.nx, gs.nz, m->half) : 0;
    d.nt = m->nt; d.si = m->si; d.nsnap = m->nsnap;
    job.first_phase_step = backward_only == 1 ? m->nt : 0;
    job.g0 = g_ - job.first_phase_step;
    job.total = modelling ? m->nt : (backward_only == 2 ? m->nt : 2 * m->nt);
    d.g0 = job.g0;
    d.total_steps = job.total;
    d.trace_nt = modelling ? m->nt : sh.nt;
    d.src_x = geo.src_x; d.src_z = geo.src_z;
    d.snap_type = snap_type();
    d.field_slot = s;
    d.nrec = sh.nrec;
    d.c0 = m->coef.c0;
    for (int k = 0; k <= kMaxHalf; ++k) { d.cx[k] = m->coef.cx[k]; d.cz[k] = m->coef.cz[k]; }
    d.vdt2 = m->vdt2.get<float>();
    d.ldz_model = m->g.ldz;
    d.wx = sl.wx.get<float>();
    d.wz = m->wz.get<float>();
    d.wavelet = m->wavelet.get<float>();
    d.traces = dev_traces ? sh.traces : sl.traces.get<float>();
    d.col_start = sl.col_start.get<int>();
    d.pts = sl.pts.get<PointEntry>();
    d.pts_ir = sl.ir.get<int>();
    d.rec_col = sl.rec_col.get<int>();
    d.rec_zs = sl.rec_z.get<int>();
    d.rec_out = sl.rec.get<float>();
    char* snap = arena_.get<char>() + snap_off;
    d.snap = snap_bytes ? snap : nullptr;
    const int sty = snap_type();
    const size_t es = sty == kSnapF64 ? 8 : (sty == kSnapF32 ? 4 : 2);
    d.snap_exp = (snap_bytes && (sty == kSnapBF16 || sty == kSnapF16))
                     ? reinterpret_cast<int8_t*>(snap + round256((size_t)m->nsnap * gs.nx * gs.lds * es))
                     : nullptr;
    if (modelling) {
        d.flags = kFlagRecord;
    } else if (backward_only == 2) {
        d.flags = kFlagSnapshots | (rec_host ? kFlagRecord : 0);   // forward() of the method API
        d.total_steps = job.total = m->nt;
    } else if (recon_) {
        d.flags = kFlagRecon | kFlagImage;
    } else {
        d.flags = (backward_only ? 0 : kFlagSnapshots) | kFlagImage;
    }
    const size_t n_acc = (size_t)gs.nx * gs.lds;
    if (cfg_.mode == RTM_B200_MODE_PLAIN || modelling) {
        d.acc_mode = kAccPlain;
        d.img = m->img.get<char>() + (size_t)sh.x0 * gs.lds * elem();
        d.ill = m->ill.get<char>() + (size_t)sh.x0 * gs.lds * elem();
    } else {
        d.acc_mode = (cfg_.accumulation == RTM_B200_ACC_COMPENSATED && !f64_) ? kAccCompensated : kAccPlain;
        char* a = sl.acc.get<char>();
        d.img = a;
        d.ill = a + n_acc * elem();
        // FP32 sums, then their BF16 compensation words (kAccCompensated)
        d.img_c = f64_ ? nullptr : a + 2 * n_acc * 4;
        d.ill_c = f64_ ? nullptr : a + 2 * n_acc * 4 + n_acc * 2;
        RTMB_CUDA(cudaMemsetAsync(a, 0, f64_ ? 2 * n_acc * 8 : 2 * n_acc * 4 + 2 * n_acc * 2, stream_));
    }
    std::memcpy(st + o_desc, &d, sizeof(ShotDesc));
    host_descs_[(size_t)s] = d;

    RTMB_CUDA(cudaMemcpyAsync(sl.wx.get(), st + o_wx, wx.size() * 4, cudaMemcpyHostToDevice, stream_));
    RTMB_CUDA(cudaMemcpyAsync(sl.col_start.get(), st + o_cs, geo.col_start.size() * 4, cudaMemcpyHostToDevice,
                              stream_));
    if (!geo.pts.empty())
        RTMB_CUDA(cudaMemcpyAsync(sl.pts.get(), st + o_pts, geo.pts.size() * sizeof(PointEntry),
                                  cudaMemcpyHostToDevice, stream_));
    if (!geo.ir.empty())
        RTMB_CUDA(cudaMemcpyAsync(sl.ir.get(), st + o_ir, geo.ir.size() * 4, cudaMemcpyHostToDevice, stream_));
    RTMB_CUDA(cudaMemcpyAsync(sl.rec_col.get(), st + o_rc, geo.rec_col.size() * 4, cudaMemcpyHostToDevice, stream_));
    if (!geo.rec_z.empty())
        RTMB_CUDA(cudaMemcpyAsync(sl.rec_z.get(), st + o_rz, geo.rec_z.size() * 4, cudaMemcpyHostToDevice, stream_));
    job.tr_wait = false;
    if (trace_h2d && pinned_traces && backward_only == 0) {
        // A full migration reads its traces from the backward pass on, nt steps
        // from now: upload them on the copy stream once the work queued so far
        // (the slot's previous job reads this buffer) is done, so they overlap
        // the forward pass; run_chunk makes the step stream wait before the
        // backward pass starts.
        RTMB_CUDA(cudaEventRecord(sl.free_ev, stream_));
        RTMB_CUDA(cudaStreamWaitEvent(copy_stream_, sl.free_ev, 0));
        RTMB_CUDA(cudaMemcpyAsync(sl.traces.get(), sh.traces, trace_h2d * 4, cudaMemcpyHostToDevice, copy_stream_));
        RTMB_CUDA(cudaEventRecord(sl.tr_ready, copy_stream_));
        job.tr_wait = true;
    } else if (trace_h2d) {
        RTMB_CUDA(cudaMemcpyAsync(sl.traces.get(), pinned_traces ? (const void*)sh.traces : (const void*)(st + o_tr),
                                  trace_h2d * 4, cudaMemcpyHostToDevice, stream_));
    }
    times.h2d_bytes += (double)trace_h2d * 4.0 +
                       (double)(wx.size() * 4 + geo.col_start.size() * 4 + geo.pts.size() * sizeof(PointEntry) +
                                geo.ir.size() * 4 + geo.rec_col.size() * 4 + geo.rec_z.size() * 4 +
                                sizeof(ShotDesc));
    RTMB_CUDA(cudaMemcpyAsync(descs_.get<ShotDesc>() + s, st + o_desc, sizeof(ShotDesc), cudaMemcpyHostToDevice,
                              stream_));
    // Columns [0, H) and [nxe - H, nxe_cap) of a job whose tile columns may
    // start at H: zero in both field levels (tiles need not cover them).
    if (job.shift_cols) {
        const size_t col = (size_t)ldz_cap_ * elem();
        const int H = m->half;
        for (int b = 0; b < 2; ++b) {
            char* fb = pool_.get<char>() + ((size_t)s * nbuf_ + b) * nxe_cap_ * ldz_cap_ * elem();
            RTMB_CUDA(cudaMemsetAsync(fb, 0, (size_t)H * col, stream_));
            RTMB_CUDA(cudaMemsetAsync(fb + (size_t)(gs.nxe - H) * col, 0, (size_t)(nxe_cap_ - gs.nxe + H) * col,
                                      stream_));
        }
    }
    // Rows outside a shifted job's bands: zero in both field levels.
    if (gs.z0 > 0) {
        const size_t pitch = (size_t)ldz_cap_ * elem();
        const int below = gs.z0 + kTileZ * gs.ntz;
        for (int b = 0; b < 2; ++b) {
            char* fb = pool_.get<char>() + ((size_t)s * nbuf_ + b) * nxe_cap_ * ldz_cap_ * elem();
            RTMB_CUDA(cudaMemset2DAsync(fb, pitch, 0, (size_t)gs.z0 * elem(), (size_t)nxe_cap_, stream_));
            if (below < ldz_cap_)
                RTMB_CUDA(cudaMemset2DAsync(fb + (size_t)below * elem(), pitch, 0, (size_t)(ldz_cap_ - below) * elem(),
                                            (size_t)nxe_cap_, stream_));
        }
    }
    // The slot's (v dt)^2 on the shot's extended grid (third field buffer).
    RTMB_TRY(share_model_vdt2(m));
    {
        char* vbuf = pool_.get<char>() + ((size_t)s * nbuf_ + 2) * nxe_cap_ * ldz_cap_ * elem();
        RTMB_CUDA(launch_slot_vdt2(vbuf, f64_, ldz_cap_, gs.nxe, m->vdt2.get<float>(), m->g.ldz, gs.nb, gs.nx,
                                   sh.x0, stream_));
        launches_ += 1;
    }
    RTMB_CUDA(cudaEventRecord(sl.staged, stream_));

    job.active = true;
    tiles_dirty_ = true;
    if (!modelling && backward_only != 2) {
        const double upd = 2.0 * m->nt * (double)gs.nxe * gs.nze;
        times.cell_updates += upd;
        const double nint = (double)gs.nx * gs.nz;
        if (recon_) {
            // the source field's reverse steps over the interior and its band,
            // the strips written forward and read backward, the image RMW
            const double rev = (double)std::max(m->nt - 2, 0) * (gs.nx + 2.0 * m->half) * (gs.nz + 2.0 * m->half);
            const double strips = 2.0 * std::max(m->nt - 1, 0) * (double)d.bsize * 4.0;
            times.algorithmic_bytes += 16.0 * (upd + rev) + strips + m->nsnap * nint * (4.0 + 16.0) +
                                       (double)sh.nrec * m->nt * 4.0;
        } else {
            const double s_b = (double)es;
            times.algorithmic_bytes += 16.0 * upd + m->nsnap * nint * s_b + m->nsnap * nint * (s_b + 16.0) +
                                       (double)sh.nrec * m->nt * 4.0;
        }
        times.shots += 1;
    }
    if (m->t_start < 0) m->t_start = clock();
    return RTM_B200_OK;
}

int Engine::finish_job(int s) {
    Job& job = jobs_[(size_t)s];
    Model* m = job.m;
    Slot& sl = slots_[(size_t)s];
    if (job.modelling || (job.rec_host && host_descs_[(size_t)s].flags & kFlagRecord)) {
        if (job.rec_host) {
            RTMB_CUDA(cudaStreamSynchronize(stream_));
            const ShotData& sh = m->shots[(size_t)job.shot];
            RTMB_CUDA(cudaMemcpy(job.rec_host, sl.rec.get(), sizeof(float) * (size_t)sh.nrec * m->nt,
                                 cudaMemcpyDeviceToHost));
        }
    } else if (cfg_.mode != RTM_B200_MODE_PLAIN && (host_descs_[(size_t)s].flags & kFlagImage)) {
        const ShotDesc& d = host_descs_[(size_t)s];
        if (f64_)
            RTMB_CUDA(launch_stack_f64((const double*)d.img, (const double*)d.ill, m->img64.get<double>(),
                                       m->ill64.get<double>(), d.nx, d.lds, job.x0, stream_));
        else
            RTMB_CUDA(launch_stack_f32((const float*)d.img, (const uint16_t*)d.img_c, (const float*)d.ill,
                                       (const uint16_t*)d.ill_c, m->img64.get<double>(), m->ill64.get<double>(), d.nx,
                                       d.lds, job.x0, stream_));
        launches_ += 1;
    }
    if (job.owns_snap && job.snap_bytes) alloc_.release(job.snap_off, job.snap_bytes);
    m->shots_done += 1;
    job.active = false;
    tiles_dirty_ = true;
    return RTM_B200_OK;
}

int Engine::retire_finished() {
    for (int s = 0; s < (int)jobs_.size(); ++s) {
        Job& j = jobs_[(size_t)s];
        if (j.active && g_ - j.g0 >= j.total) RTMB_TRY(finish_job(s));
    }
    return RTM_B200_OK;
}

int Engine::build_tiles() {
    std::vector<long long> sig;
    std::map<int, std::vector<TileRef>> by_half;
    for (int s = 0; s < (int)jobs_.size(); ++s) {
        const Job& j = jobs_[(size_t)s];
        if (!j.active) continue;
        const int TX = step_tile_x(variant(j.m->half));
        const int H0 = j.m->half;
        const int ntx0 = (j.gs.nxe + TX - 1) / TX, ntx1 = (j.gs.nxe - 2 * H0 + TX - 1) / TX;
        const int cx0 = j.shift_cols && ntx1 < ntx0 ? H0 : 0;   // first column of the tile columns
        const int ntx = cx0 ? ntx1 : ntx0;
        std::vector<uint8_t> tflags((size_t)ntx * j.gs.ntz, 0);
        for (const auto& c : j.rec_cells)
            tflags[(size_t)((c.first - cx0) / TX) * j.gs.ntz + (c.second - j.gs.z0) / kTileZ] = 1;
        auto& vec = by_half[j.m->half];
        const ShotDesc& d = host_descs_[(size_t)s];
        // Reconstruction: tiles holding band cells store the strips forward; the
        // source field's own tiles cover the interior and its band.
        const int H = j.m->half, nb = j.gs.nb;
        auto meets = [&](int tx, int tz, int xa, int xb, int za, int zb) {
            return tx * TX < xb && tx * TX + TX > xa && tz * kTileZ < zb && tz * kTileZ + kTileZ > za;
        };
        const bool rec = (d.flags & kFlagRecon) != 0;
        // Tiles whose columns all lie inside the aperture window load (v dt)^2
        // from the model's shared table (the same values as the slot's copy).
        const bool shared_vd = !f64_ && shared_vd_uid_ != 0 && j.m->uid == shared_vd_uid_;
        auto place_vd = [&](TileRef r) {
            if (shared_vd && r.x0 >= d.nb && r.x0 + TX <= d.nb + d.win_nx) {
                r.vd_x = r.x0 - d.nb + d.model_x0;
                r.vd_buf = shared_vd_buf();
            }
            return r;
        };
        for (int tz = 0; tz < j.gs.ntz; ++tz)
            for (int tx = 0; tx < ntx; ++tx) {
                TileRef r = place_vd(make_tile_ref(d, s, tx, tz, TX, tflags[(size_t)tx * j.gs.ntz + tz] != 0, nbuf_,
                                                   false, j.gs.z0, cx0));
                if (rec && (meets(tx, tz, nb - H, nb, nb, nb + j.gs.nz) ||
                            meets(tx, tz, nb + j.gs.nx, nb + j.gs.nx + H, nb, nb + j.gs.nz) ||
                            meets(tx, tz, nb, nb + j.gs.nx, nb - H, nb) ||
                            meets(tx, tz, nb, nb + j.gs.nx, nb + j.gs.nz, nb + j.gs.nz + H)))
                    r.flags |= kFlagBandTile;
                vec.push_back(r);
            }
        if (rec)
            for (int tz = 0; tz < j.gs.ntz; ++tz)
                for (int tx = 0; tx < ntx; ++tx)
                    if (meets(tx, tz, nb - H, nb + j.gs.nx + H, nb - H, nb + j.gs.nz + H))
                        vec.push_back(place_vd(make_tile_ref(d, s, tx, tz, TX, false, nbuf_, true)));
        sig.push_back(s);
        sig.push_back(j.m->half);
        sig.push_back(ntx);
        sig.push_back(j.gs.ntz);
        sig.push_back(j.gs.z0);
        sig.push_back(cx0);
        sig.push_back(j.g0);
        sig.push_back(j.total);
        sig.push_back(d.flags);
        sig.push_back(shared_vd ? shared_vd_buf() : -1);
    }
    sig.push_back(tile_x_);
    sig.push_back(warps_);
    sig.push_back(spare_);
    sig.push_back(exact() ? 1 : 0);
    sig.push_back(stage_override_);
    sig.push_back(kind_);
    sig.push_back(march_m_);
    tiles_dirty_ = false;
    if (sig == tile_sig_) return RTM_B200_OK;
    tile_sig_ = sig;
    groups_.clear();
    std::vector<TileRef> all;
    for (auto& kv : by_half) {
        groups_.push_back(Group{kv.first, (int)all.size(), (int)kv.second.size()});
        all.insert(all.end(), kv.second.begin(), kv.second.end());
    }
    if (all.empty()) return RTM_B200_OK;
    // The device tile list may still be read by queued launches: wait for them.
    RTMB_CUDA(cudaStreamSynchronize(stream_));
    // Room for every slot's largest tile count (16-column tiles over the pool's
    // width), so that a wider shot mix does not regrow the list mid-run.
    const size_t most = (size_t)nslots_ * (recon_ ? 2 : 1) * (size_t)((nxe_cap_ + 15) / 16) *
                        (size_t)((ldz_cap_ + kTileZ - 1) / kTileZ);
    RTMB_CUDA(tiles_.reserve(std::max(all.size(), most) * sizeof(TileRef)));
    RTMB_CUDA(cudaMemcpy(tiles_.get(), all.data(), all.size() * sizeof(TileRef), cudaMemcpyHostToDevice));
    for (auto& g : groups_) {
        if (!step_variant_supported(variant(g.half)))
            return fail(RTM_B200_EUNSUPPORTED, "tile width " + std::to_string(tile_x_) + " does not fit shared memory "
                        "for this stencil order and precision (use tile_cols 0 or 16)");
        const int mk = g.half * 64 + tile_x_;
        if (variant(g.half).kind == kStepRing && !maps_.count(mk)) {
            MapPair mp;
            RTMB_TRY(encode_map(g.half, true, &mp.pc));
            RTMB_TRY(encode_map(g.half, false, &mp.box));
            maps_[mk] = mp;
        }
        RTMB_CUDA(prepare_step(variant(g.half)));
    }
    return RTM_B200_OK;
}

// The job mix a tuning result applies to: stencil half-orders present, tile
// rows of the tallest shot, and the number of shots in flight (bucketed).
std::vector<long long> Engine::tune_key() const {
    std::vector<long long> k;
    int n = 0, ntz = 0;
    std::map<int, int> halves;
    for (const auto& j : jobs_)
        if (j.active) {
            ++n;
            ntz = std::max(ntz, j.gs.ntz);
            halves[j.m->half] += 1;
        }
    for (auto& h : halves) k.push_back(h.first);
    k.push_back(ntz);
    int b = 1;
    while (b < n) b *= 2;
    k.push_back(b);
    k.push_back(f64_ ? 1 : 0);
    k.push_back(exact() ? 1 : 0);
    return k;
}

// After a failed run: drop every job, free its snapshot range and put the
// device step counter back in step with the host.
void Engine::abort_jobs() {
    cudaStreamSynchronize(copy_stream_);
    cudaStreamSynchronize(stream_);
    cudaGetLastError();
    for (auto& j : jobs_) {
        if (j.active && j.owns_snap && j.snap_bytes) alloc_.release(j.snap_off, j.snap_bytes);
        j.active = false;
    }
    tiles_dirty_ = true;
    tile_sig_.clear();
    if (graph_) { cudaGraphExecDestroy(graph_); graph_ = nullptr; }
    graph_sig_.clear();
    if (counter_.get()) {
        cudaMemcpy(counter_.get(), &g_, sizeof(long long), cudaMemcpyHostToDevice);
    }
}

// Advances every job in flight by `steps` time steps.  With autotuning on
// (tile_cols 0), the first chunk of a job mix not seen before is split: each
// candidate (columns per warp, pipeline stages) runs a few real steps timed with
// CUDA events, and the fastest is kept for the mix.  Every candidate computes
// identical cells, so tuning costs no work.
int Engine::run_chunk(int steps) {
    // Traces uploading on the copy stream must land before their job's backward
    // pass, which may start inside this chunk.
    for (size_t s = 0; s < jobs_.size(); ++s) {
        Job& j = jobs_[s];
        if (j.active && j.tr_wait && g_ + steps > j.g0 + j.m->nt) {
            RTMB_CUDA(cudaStreamWaitEvent(stream_, slots_[s].tr_ready, 0));
            j.tr_wait = false;
        }
    }
    if (!autotune_ || steps <= 0) return run_steps(steps);
    if (tiles_dirty_ || groups_.empty()) {
        const std::vector<long long> key = tune_key();
        auto hit = tuned_.find(key);
        auto apply = [&](const TuneChoice& c) {
            if (kind_ != c.kind || warps_ != c.warps || tile_x_ != c.tile_x || stage_override_ != c.stages ||
                march_m_ != c.march_m || spare_ != c.spare)
                tiles_dirty_ = true;
            kind_ = c.kind;
            warps_ = c.warps;
            spare_ = c.spare;
            tile_x_ = c.tile_x;
            stage_override_ = c.stages;
            march_m_ = c.march_m;
        };
        if (hit != tuned_.end()) {
            apply(hit->second);
        } else {
            // Ring shapes (consumer warps x tile width, default stages) and the
            // register-march strip lengths.  The march kernel's FMA arithmetic
            // is not the ring kernel's, so with FMA it is not a candidate: every
            // candidate of a mix must compute the same cells.
            // spare = 1: the grid leaves one CTA slot per SM free, so the next
            // (programmatic dependent) step's CTAs are resident and waiting
            // before this step ends: it pays when steps are short.
            std::vector<TuneChoice> cands = {{kStepRing, 4, 16, 0, 3, 0}, {kStepRing, 4, 16, 0, 3, 1},
                                             {kStepRing, 8, 16, 0, 3, 0}, {kStepRing, 8, 16, 0, 3, 1},
                                             {kStepRing, 8, 32, 0, 3, 0}};
            if (exact() && !shifted_bands())
                for (int m : {2, 3, 5}) cands.push_back({kStepMarch, 8, 16, 0, m, 0});
            if (pin_kind_ >= 0) {
                std::vector<TuneChoice> keep;
                for (const auto& c : cands)
                    if (c.kind == pin_kind_) keep.push_back(c);
                cands.swap(keep);
            }
            // Two interleaved rounds of k timed steps per candidate; a
            // candidate's time is its faster round, so one disturbed sample
            // cannot decide the pick.
            const int ncand = (int)cands.size();
            const int k = std::min(12, steps / std::max(2 * ncand, 1));
            if (k >= 4) {
                TuneRecord rec;
                rec.key = key;
                std::map<int, int> halves;
                for (const auto& j : jobs_)
                    if (j.active) halves[j.m->half] = 1;
                std::vector<double> best_us((size_t)ncand, 1e300);
                for (int round = 0; round < 2; ++round)
                    for (int ci = 0; ci < ncand; ++ci) {
                        const TuneChoice& c = cands[(size_t)ci];
                        apply(c);
                        bool ok = true;   // e.g. FP64 order-12 tiles of 32 columns exceed shared memory
                        for (const auto& h : halves) ok = ok && step_variant_supported(variant(h.first));
                        if (!ok || (f64_ && c.kind == kStepMarch)) continue;
                        tiles_dirty_ = true;
                        RTMB_CUDA(cudaStreamSynchronize(stream_));
                        RTMB_TRY(build_tiles());
                        RTMB_CUDA(cudaEventRecord(tune_ev0_, stream_));
                        RTMB_TRY(run_steps(k));
                        RTMB_CUDA(cudaEventRecord(tune_ev1_, stream_));
                        RTMB_CUDA(cudaEventSynchronize(tune_ev1_));
                        float ms = 0.f;
                        RTMB_CUDA(cudaEventElapsedTime(&ms, tune_ev0_, tune_ev1_));
                        best_us[(size_t)ci] = std::min(best_us[(size_t)ci], 1e3 * ms / k);
                        steps -= k;
                    }
                TuneChoice pick = cands[0];
                double best = 1e300;
                for (int ci = 0; ci < ncand; ++ci) {
                    rec.cands.push_back(cands[(size_t)ci]);
                    const double us = best_us[(size_t)ci] < 1e299 ? best_us[(size_t)ci] : -1.0;
                    rec.us_per_step.push_back(us);
                    if (us > 0 && us < best) { best = us; pick = cands[(size_t)ci]; }
                }
                apply(pick);
                rec.pick = pick;
                tuned_[key] = pick;
                tune_log_.push_back(rec);
                tiles_dirty_ = true;
            }
        }
    }
    return run_steps(steps);
}

int Engine::run_steps(int steps) {
    if (tiles_dirty_) RTMB_TRY(build_tiles());
    if (groups_.empty() || steps <= 0) return RTM_B200_OK;
    auto enqueue = [&]() -> int {
        for (int j = 0; j < steps; ++j)
            for (const Group& g : groups_) {
                const StepVariant v = variant(g.half);
                StepParams p{};
                p.fields = pool_.get();
                p.buf_stride = (long long)nxe_cap_ * ldz_cap_;
                p.slot_stride = nbuf_ * p.buf_stride;
                p.nbuf = nbuf_;
                p.ldz = ldz_cap_;
                p.ntiles = g.count;
                p.descs = descs_.get<ShotDesc>();
                p.tiles = tiles_.get<TileRef>() + g.offset;
                p.step_counter = counter_.get<long long>();
                p.step_offset = j;
                p.error_word = errword_.get<int>();
                p.pdl = 1;
                p.stall_tile = -1;
                if (stall_tile_ >= 0 && j == 0) {
                    p.stall_tile = stall_tile_;
                    stall_tile_ = -1;
                }
                p.march_m = v.march_m;
                static const MapPair kNoMaps{};
                const MapPair& mp = v.kind == kStepRing ? maps_[g.half * 64 + tile_x_] : kNoMaps;
                RTMB_CUDA(launch_step(v, mp.pc, mp.box, p, stream_));
            }
        RTMB_CUDA(launch_advance_counter(counter_.get<long long>(), steps, stream_));
        return RTM_B200_OK;
    };
    cudaEvent_t& slot_ev = chunk_ev_[chunk_k_ % kChunksInFlight];
    if (chunk_k_ >= kChunksInFlight) RTMB_CUDA(cudaEventSynchronize(slot_ev));
    const bool use_graph = cfg_.chunk_steps >= 0 && stall_tile_ < 0;
    if (use_graph) {
        if (!graph_ || graph_sig_ != tile_sig_ || graph_steps_ != steps) {
            if (graph_) { cudaGraphExecDestroy(graph_); graph_ = nullptr; }
            cudaGraph_t gr = nullptr;
            RTMB_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
            const int rc = enqueue();
            const cudaError_t ce = cudaStreamEndCapture(stream_, &gr);
            if (rc != RTM_B200_OK) { if (gr) cudaGraphDestroy(gr); return rc; }
            RTMB_CUDA(ce);
            const cudaError_t ie = cudaGraphInstantiate(&graph_, gr, 0);
            cudaGraphDestroy(gr);
            RTMB_CUDA(ie);
            graph_sig_ = tile_sig_;
            graph_steps_ = steps;
        }
        RTMB_CUDA(cudaGraphLaunch(graph_, stream_));
    } else {
        RTMB_TRY(enqueue());
    }
    RTMB_CUDA(cudaEventRecord(slot_ev, stream_));
    ++chunk_k_;
    launches_ += steps * (int)groups_.size() + 1;
    g_ += steps;
    return RTM_B200_OK;
}

int Engine::chunk_for(const Model& m) const {
    int target = cfg_.chunk_steps > 0 ? cfg_.chunk_steps : 256;
    if (cfg_.mode == RTM_B200_MODE_PLAIN) {
        // chunks that tile both passes of one shot with little overrun
        const int per_pass = m.nt;
        const int k = (per_pass + target - 1) / target;
        return (per_pass + k - 1) / k;
    }
    return cfg_.chunk_steps > 0 ? cfg_.chunk_steps : 64;
}

int Engine::check_device_error() {
    int e = 0;
    RTMB_CUDA(cudaStreamSynchronize(stream_));
    RTMB_CUDA(cudaMemcpy(&e, errword_.get(), sizeof(int), cudaMemcpyDeviceToHost));
    if (e) {
        cudaMemset(errword_.get(), 0, sizeof(int));
        return fail(RTM_B200_ETIMEOUT, "a bounded device-side wait gave up (error bits " + std::to_string(e) + ")");
    }
    return RTM_B200_OK;
}

int Engine::admit_from(std::deque<std::pair<Model*, int>>& q, bool modelling, float* rec_base,
                       const std::vector<size_t>* rec_offsets, int* admitted, int limit) {
    *admitted = 0;
    while (!q.empty() && (limit < 0 || *admitted < limit)) {
        int free_slot = -1;
        for (int s = 0; s < nslots_; ++s)
            if (!jobs_[(size_t)s].active) { free_slot = s; break; }
        if (free_slot < 0) break;
        Model* m = q.front().first;
        const int shot = q.front().second;
        const ShotData& sh = m->shots[(size_t)shot];
        const GridDims gs = make_grid(sh.wnx, m->g.nz, m->g.nb, m->half);
        if (gs.nxe > nxe_cap_ || m->g.ldz > ldz_cap_) return fail(RTM_B200_EINVAL, "shot grid exceeds the field pool");
        size_t off = 0, bytes = 0;
        if (!modelling) {
            bytes = snap_alloc_bytes(*m, gs);
            if (!alloc_.allocate(bytes, &off)) break;
        }
        float* rec = modelling && rec_base ? rec_base + (*rec_offsets)[(size_t)shot] : nullptr;
        const int rc = start_job(free_slot, m, shot, modelling, rec, 0, off, bytes, true);
        if (rc != RTM_B200_OK) {
            if (bytes) alloc_.release(off, bytes);
            return rc;
        }
        q.pop_front();
        *admitted += 1;
    }
    return RTM_B200_OK;
}

int Engine::run_queue(std::deque<std::pair<Model*, int>>& q, bool modelling, float* rec_base,
                      const std::vector<size_t>* rec_offsets) {
    // Plain migration with two slots runs shots staggered by one pass: shot s+1
    // is admitted when shot s starts its backward pass, so s+1's forward pass
    // overlaps s's backward pass and s+1 images only after s has finished.  Every
    // image cell still receives its terms in the reference's shot and step order
    // (bit for bit), and each step launch carries two shots' tiles.
    const bool staggered = cfg_.mode == RTM_B200_MODE_PLAIN && !modelling && nslots_ > 1;
    while (true) {
        RTMB_TRY(retire_finished());
        int admitted = 0;
        if (staggered) {
            bool in_backward = true;
            for (const auto& j : jobs_)
                if (j.active && g_ - j.g0 < j.m->nt) in_backward = false;
            if (in_backward) RTMB_TRY(admit_from(q, modelling, rec_base, rec_offsets, &admitted, 1));
        } else {
            RTMB_TRY(admit_from(q, modelling, rec_base, rec_offsets, &admitted));
        }
        if (active_jobs() == 0) {
            if (!q.empty()) return fail(RTM_B200_ENOMEM, "a shot does not fit the device memory budget");
            break;
        }
        int remaining = 0, next_event = INT_MAX;
        for (const auto& j : jobs_) {
            if (!j.active) continue;
            const int done = (int)(g_ - j.g0);
            remaining = std::max(remaining, j.total - done);
            next_event = std::min(next_event, j.total - done);
            if (!q.empty() && done < j.m->nt) next_event = std::min(next_event, j.m->nt - done);
        }
        const int c = chunk_for(*jobs_[0].m);
        RTMB_TRY(run_chunk(std::min(c, staggered ? next_event : remaining)));
    }
    return RTM_B200_OK;
}

int Engine::zero_model_images(Model& m) {
    const size_t n = (size_t)m.g.nx * m.g.lds;
    if (cfg_.mode == RTM_B200_MODE_PLAIN) {
        RTMB_CUDA(m.img.reserve(n * elem()));
        RTMB_CUDA(m.ill.reserve(n * elem()));
        RTMB_CUDA(cudaMemsetAsync(m.img.get(), 0, n * elem(), stream_));
        RTMB_CUDA(cudaMemsetAsync(m.ill.get(), 0, n * elem(), stream_));
    } else {
        RTMB_CUDA(m.img64.reserve(n * 8));
        RTMB_CUDA(m.ill64.reserve(n * 8));
        RTMB_CUDA(cudaMemsetAsync(m.img64.get(), 0, n * 8, stream_));
        RTMB_CUDA(cudaMemsetAsync(m.ill64.get(), 0, n * 8, stream_));
    }
    return RTM_B200_OK;
}

int Engine::finalize_model_image(Model& m, float* img, float* ill, double* img64, double* ill64) {
    const GridDims& g = m.g;
    const size_t n = (size_t)g.nx * g.nz;
    const int row0 = g.nb - g.zs0;
    DevMem tmp;
    RTMB_CUDA(tmp.alloc(n * 8 * 2));
    const bool plain = cfg_.mode == RTM_B200_MODE_PLAIN;
    const bool src64 = !plain || f64_;
    const void* si = plain ? m.img.get() : m.img64.get();
    const void* ss = plain ? m.ill.get() : m.ill64.get();
    if (img || ill) {
        float* d = tmp.get<float>();
        if (src64) {
            RTMB_CUDA(launch_extract_f64_to_f32((const double*)si, g.lds, row0, d, g.nx, g.nz, stream_));
            RTMB_CUDA(launch_extract_f64_to_f32((const double*)ss, g.lds, row0, d + n, g.nx, g.nz, stream_));
        } else {
            RTMB_CUDA(launch_extract_f32((const float*)si, g.lds, row0, d, g.nx, g.nz, 1, stream_));
            RTMB_CUDA(launch_extract_f32((const float*)ss, g.lds, row0, d + n, g.nx, g.nz, 1, stream_));
        }
        if (img) RTMB_CUDA(cudaMemcpyAsync(img, d, n * 4, cudaMemcpyDefault, stream_));
        if (ill) RTMB_CUDA(cudaMemcpyAsync(ill, d + n, n * 4, cudaMemcpyDefault, stream_));
        times.d2h_bytes += (double)n * 4 * ((img && !is_device_ptr(img)) + (ill && !is_device_ptr(ill)));
        RTMB_CUDA(cudaStreamSynchronize(stream_));
    }
    if (img64 || ill64) {
        double* d = tmp.get<double>();
        if (src64) {
            RTMB_CUDA(launch_extract_f64((const double*)si, g.lds, row0, d, g.nx, g.nz, stream_));
            RTMB_CUDA(launch_extract_f64((const double*)ss, g.lds, row0, d + n, g.nx, g.nz, stream_));
        } else {
            float* f = reinterpret_cast<float*>(d + n);   // second half as float scratch
            RTMB_CUDA(launch_extract_f32((const float*)si, g.lds, row0, f, g.nx, g.nz, 1, stream_));
            RTMB_CUDA(launch_widen(f, d, n, stream_));
            RTMB_CUDA(launch_extract_f32((const float*)ss, g.lds, row0, f, g.nx, g.nz, 1, stream_));
            RTMB_CUDA(launch_widen(f, d + n, n, stream_));
        }
        if (img64) RTMB_CUDA(cudaMemcpyAsync(img64, d, n * 8, cudaMemcpyDefault, stream_));
        if (ill64) RTMB_CUDA(cudaMemcpyAsync(ill64, d + n, n * 8, cudaMemcpyDefault, stream_));
        times.d2h_bytes += (double)n * 8 * ((img64 && !is_device_ptr(img64)) + (ill64 && !is_device_ptr(ill64)));
        RTMB_CUDA(cudaStreamSynchronize(stream_));
    }
    launches_ += 4;
    return RTM_B200_OK;
}

// ------------------------------------------------------------ migrate etc.
int Engine::migrate(const rtm_b200_shot* shots, int nshots, float* img, float* ill, double* img64,
                    double* ill64) {
    if (!model_) return fail(RTM_B200_ESTATE, "migrate before setup");
    RTMB_CUDA(cudaSetDevice(device_));
    const auto t_start = std::chrono::steady_clock::now();
    Model& m = *model_;
    RTMB_TRY(copy_shots(m, shots, nshots, true));
    keep_snap_ = false;

    // Memory plan: field pool slots + snapshot arena inside the budget.
    const GridDims& g = m.g;
    size_t freeb = 0, totalb = 0;
    RTMB_CUDA(cudaStreamSynchronize(stream_));
    RTMB_CUDA(cudaMemGetInfo(&freeb, &totalb));
    // memory the engine already holds counts towards the budget it may use
    const size_t held = pool_.bytes() + arena_.bytes();
    const size_t budget = cfg_.device_mem_budget > 0 ? (size_t)cfg_.device_mem_budget
                                                     : (size_t)(0.9 * (double)(freeb + held));
    size_t snap_max = 0, snap_sum = 0;
    for (auto& sh : m.shots) {
        const size_t b = snap_alloc_bytes(m, make_grid(sh.wnx, g.nz, g.nb, m.half));
        snap_max = std::max(snap_max, b);
        snap_sum += b;
    }
    const size_t per_slot = (size_t)(nbuf_ - 1) * g.nxe * g.ldz * elem() + (size_t)g.nx * g.lds * 16 +
                            (size_t)4 * g.nxe * 3 + (size_t)m.nt * 4 * 2048;
    int want = 1;
    if (cfg_.mode == RTM_B200_MODE_PLAIN && nshots > 1 &&
        2 * (per_slot + snap_max) + ((size_t)512 << 20) <= budget)
        want = 2;   // two shots staggered by one pass (run_queue)
    InflightTune* tuning = nullptr;
    int tuning_cand = -1;
    if (cfg_.mode != RTM_B200_MODE_PLAIN) {
        const size_t snap_avg = nshots > 0 ? snap_sum / (size_t)nshots : snap_max;
        const size_t fit = budget / std::max<size_t>(per_slot + snap_avg, 1);
        if (cfg_.max_shots_in_flight > 0) {
            want = cfg_.max_shots_in_flight;
        } else {
            // Tuned across calls: the candidates that fit memory and the survey
            // run one per call on real work; then the fastest is kept.
            const std::vector<long long> key = {g.nx, g.nz, m.half, m.nt, snap_type(), nshots};
            for (auto& t : inflight_log_)
                if (t.key == key) tuning = &t;
            if (!tuning) {
                InflightTune t;
                t.key = key;
                for (int c : {16, 32, 48, 64})
                    if ((size_t)c <= fit && c <= std::max(nshots, 1)) t.cands.push_back(c);
                if (t.cands.empty()) t.cands.push_back((int)std::max<size_t>(1, std::min<size_t>(fit, 16)));
                t.shots_per_s.assign(t.cands.size(), 0.0);
                if (t.cands.size() == 1) t.pick = t.cands[0];
                inflight_log_.push_back(t);
                tuning = &inflight_log_.back();
            }
            if (tuning->pick) {
                want = tuning->pick;
                tuning = nullptr;
            } else {
                for (size_t c = 0; c < tuning->cands.size(); ++c)
                    if (tuning->shots_per_s[c] == 0.0) { tuning_cand = (int)c; break; }
                want = tuning->cands[(size_t)tuning_cand];
            }
        }
        want = std::min(want, std::max(nshots, 1));
        want = (int)std::max<size_t>(1, std::min<size_t>((size_t)want, fit));
    }
    RTMB_TRY(ensure_pool(want, g.nxe, g.ldz));
    size_t arena = cfg_.mode == RTM_B200_MODE_PLAIN ? (size_t)want * snap_max
                                                    : (budget > (size_t)want * per_slot ? budget - (size_t)want * per_slot : 0);
    arena = std::max(arena, snap_max);
    // Keep the current store when it is big enough and not grossly oversized.
    const bool keep_arena = arena_.bytes() >= arena && arena_.bytes() <= arena + arena / 4 + ((size_t)1 << 30);
    if (!keep_arena) {
        arena_.release();
        RTMB_CUDA(cudaMemGetInfo(&freeb, &totalb));
        arena = std::min(arena, freeb > ((size_t)256 << 20) ? freeb - ((size_t)256 << 20) : 0);
        if (arena < snap_max)
            return fail(RTM_B200_ENOMEM, "snapshot store for one shot does not fit device memory");
        cudaError_t e = arena_.alloc(arena);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(RTM_B200_ENOMEM, "cannot allocate the snapshot store");
        }
    }
    alloc_.reset(arena_.bytes());
    RTMB_TRY(zero_model_images(m));

    std::deque<std::pair<Model*, int>> q;
    for (int i = 0; i < nshots; ++i) q.emplace_back(&m, i);
    const int launches0 = launches_;
    RTMB_CUDA(cudaEventRecord(ev0_, stream_));
    if (const int rc = run_queue(q, false, nullptr, nullptr); rc != RTM_B200_OK) {
        abort_jobs();
        return rc;
    }
    RTMB_TRY(retire_finished());
    RTMB_CUDA(cudaEventRecord(ev1_, stream_));
    RTMB_TRY(check_device_error());
    float ms = 0;
    RTMB_CUDA(cudaEventElapsedTime(&ms, ev0_, ev1_));
    times.kernel += ms * 1e-3;
    if (tuning && ms > 0) {
        tuning->shots_per_s[(size_t)tuning_cand] = nshots / (ms * 1e-3);
        bool all = true;
        for (double r : tuning->shots_per_s) all = all && r > 0.0;
        if (all) {
            size_t b = 0;
            for (size_t c = 1; c < tuning->cands.size(); ++c)
                if (tuning->shots_per_s[c] > tuning->shots_per_s[b]) b = c;
            tuning->pick = tuning->cands[b];
        }
    }
    const auto t_d2h = std::chrono::steady_clock::now();
    stack_ready_ = true;
    RTMB_TRY(finalize_model_image(m, img, ill, img64, ill64));
    const auto t_end = std::chrono::steady_clock::now();
    times.d2h += std::chrono::duration<double>(t_end - t_d2h).count();
    times.total += std::chrono::duration<double>(t_end - t_start).count();
    times.kernel_launches += launches_ - launches0;
    return RTM_B200_OK;
}

int Engine::model_shots(const rtm_b200_shot* shots, int nshots, float* out) {
    if (!model_) return fail(RTM_B200_ESTATE, "model_shot before setup");
    if (!out && nshots > 0) return fail(RTM_B200_EINVAL, "output trace buffer is null");
    RTMB_CUDA(cudaSetDevice(device_));
    Model& m = *model_;
    RTMB_TRY(copy_shots(m, shots, nshots, false));
    keep_snap_ = false;
    struct ModellingScope {   // IEEE arithmetic for the duration of the call (AUTO)
        Engine* e;
        explicit ModellingScope(Engine* en) : e(en) { e->modelling_now_ = true; e->tiles_dirty_ = true; }
        ~ModellingScope() { e->modelling_now_ = false; e->tiles_dirty_ = true; }
    } scope(this);
    std::vector<size_t> offs((size_t)nshots);
    size_t acc = 0;
    for (int i = 0; i < nshots; ++i) {
        offs[(size_t)i] = acc;
        acc += (size_t)m.shots[(size_t)i].nrec * m.nt;
    }
    int want = cfg_.mode == RTM_B200_MODE_PLAIN ? 1 : std::max(1, std::min(nshots, 64));
    RTMB_TRY(ensure_pool(want, m.g.nxe, m.g.ldz));
    if (!arena_.get()) alloc_.reset(0);
    std::deque<std::pair<Model*, int>> q;
    for (int i = 0; i < nshots; ++i) q.emplace_back(&m, i);
    const int launches0 = launches_;
    if (const int rc = run_queue(q, true, out, &offs); rc != RTM_B200_OK) {
        abort_jobs();
        return rc;
    }
    RTMB_TRY(retire_finished());
    RTMB_TRY(check_device_error());
    times.kernel_launches += launches_ - launches0;
    return RTM_B200_OK;
}

int Engine::forward(const rtm_b200_shot* shot, float* snaps, float* rec) {
    if (!model_) return fail(RTM_B200_ESTATE, "forward before setup");
    if (cfg_.mode != RTM_B200_MODE_PLAIN) return fail(RTM_B200_EUNSUPPORTED, "forward() needs the plain engine");
    if (snaps && snap_type() != kSnapF32)
        return fail(RTM_B200_EUNSUPPORTED, "host snapshot exchange needs FP32 snapshots");
    RTMB_CUDA(cudaSetDevice(device_));
    Model& m = *model_;
    RTMB_TRY(copy_shots(m, shot, 1, false));
    RTMB_TRY(ensure_pool(1, m.g.nxe, m.g.ldz));
    const size_t bytes = snap_alloc_bytes(m, m.g);
    if (arena_.bytes() < bytes) {
        arena_.release();
        if (arena_.alloc(bytes) != cudaSuccess) { cudaGetLastError(); return fail(RTM_B200_ENOMEM, "snapshot store"); }
    }
    alloc_.reset(arena_.bytes());
    size_t off = 0;
    alloc_.allocate(bytes, &off);
    if (rec) RTMB_CUDA(slots_[0].rec.reserve(sizeof(float) * (size_t)std::max(shot->nrec, 1) * m.nt));
    RTMB_TRY(start_job(0, &m, 0, false, rec, 2, off, bytes, false));
    while (jobs_[0].active) {
        RTMB_TRY(run_chunk(std::min(chunk_for(m), (int)(jobs_[0].total - (g_ - jobs_[0].g0)))));
        if (g_ - jobs_[0].g0 >= jobs_[0].total) {
            RTMB_TRY(finish_job(0));
        }
    }
    RTMB_TRY(check_device_error());
    if (snaps) {
        DevMem tmp;
        const size_t n = (size_t)m.nsnap * m.g.nx * m.g.nz;
        RTMB_CUDA(tmp.alloc(n * 4));
        RTMB_CUDA(launch_extract_f32(reinterpret_cast<const float*>(arena_.get<char>() + off), m.g.lds,
                                     m.g.nb - m.g.zs0, tmp.get<float>(), m.g.nx, m.g.nz, m.nsnap, stream_));
        RTMB_CUDA(cudaStreamSynchronize(stream_));
        RTMB_CUDA(cudaMemcpy(snaps, tmp.get(), n * 4, cudaMemcpyDeviceToHost));
    }
    keep_snap_ = true;
    keep_snap_off_ = off;
    keep_snap_bytes_ = bytes;
    return RTM_B200_OK;
}

int Engine::backward(const rtm_b200_shot* shot, const float* snaps, float* img, float* ill) {
    if (!model_) return fail(RTM_B200_ESTATE, "backward before setup");
    if (cfg_.mode != RTM_B200_MODE_PLAIN) return fail(RTM_B200_EUNSUPPORTED, "backward() needs the plain engine");
    if (!img || !ill) return fail(RTM_B200_EINVAL, "image/illumination buffers are null");
    if (!snaps && !keep_snap_) return fail(RTM_B200_ESTATE, "no device snapshots: call forward first or pass them");
    if (snaps && snap_type() != kSnapF32)
        return fail(RTM_B200_EUNSUPPORTED, "host snapshot exchange needs FP32 snapshots");
    if (f64_) return fail(RTM_B200_EUNSUPPORTED, "backward() with a host image needs an FP32 engine");
    RTMB_CUDA(cudaSetDevice(device_));
    Model& m = *model_;
    RTMB_TRY(copy_shots(m, shot, 1, true));
    if (m.shots[0].wnx != m.g.nx) return fail(RTM_B200_EUNSUPPORTED, "backward() migrates on the whole model");
    RTMB_TRY(ensure_pool(1, m.g.nxe, m.g.ldz));
    const size_t bytes = snap_alloc_bytes(m, m.g);
    size_t off = keep_snap_off_;
    const size_t n = (size_t)m.g.nx * m.g.nz;
    DevMem tmp;
    if (snaps) {
        if (arena_.bytes() < bytes) {
            arena_.release();
            if (arena_.alloc(bytes) != cudaSuccess) { cudaGetLastError(); return fail(RTM_B200_ENOMEM, "snapshot store"); }
        }
        off = 0;
        RTMB_CUDA(tmp.alloc(n * m.nsnap * 4));
        RTMB_CUDA(cudaMemcpy(tmp.get(), snaps, n * m.nsnap * 4, cudaMemcpyHostToDevice));
        RTMB_CUDA(launch_insert_f32(tmp.get<float>(), m.g.nx, m.g.nz,
                                    reinterpret_cast<float*>(arena_.get<char>() + off), m.g.lds, m.g.nb - m.g.zs0,
                                    m.nsnap, stream_));
    }
    // current image/illumination become the running accumulators
    RTMB_TRY(zero_model_images(m));
    DevMem tin;
    RTMB_CUDA(tin.alloc(n * 4 * 2));
    RTMB_CUDA(cudaMemcpyAsync(tin.get(), img, n * 4, cudaMemcpyHostToDevice, stream_));
    RTMB_CUDA(cudaMemcpyAsync(tin.get<float>() + n, ill, n * 4, cudaMemcpyHostToDevice, stream_));
    RTMB_CUDA(launch_insert_f32(tin.get<float>(), m.g.nx, m.g.nz, m.img.get<float>(), m.g.lds, m.g.nb - m.g.zs0, 1,
                                stream_));
    RTMB_CUDA(launch_insert_f32(tin.get<float>() + n, m.g.nx, m.g.nz, m.ill.get<float>(), m.g.lds,
                                m.g.nb - m.g.zs0, 1, stream_));
    RTMB_TRY(start_job(0, &m, 0, false, nullptr, 1, off, bytes, false));
    while (jobs_[0].active) {
        RTMB_TRY(run_chunk(std::min(chunk_for(m), (int)(jobs_[0].total - (g_ - jobs_[0].g0)))));
        if (g_ - jobs_[0].g0 >= jobs_[0].total) RTMB_TRY(finish_job(0));
    }
    RTMB_TRY(check_device_error());
    RTMB_TRY(finalize_model_image(m, img, ill, nullptr, nullptr));
    return RTM_B200_OK;
}

int Engine::memory_probe(size_t bytes, int iters, double* gbps) {
    if (!gbps || bytes < 4096 || iters < 1) return fail(RTM_B200_EINVAL, "probe needs >= 4 KiB and >= 1 iteration");
    RTMB_CUDA(cudaSetDevice(device_));
    DevMem buf;
    const size_t half = (bytes / 2) & ~(size_t)15;
    if (buf.alloc(2 * half) != cudaSuccess) {
        cudaGetLastError();
        return fail(RTM_B200_ENOMEM, "probe buffer");
    }
    RTMB_CUDA(cudaMemsetAsync(buf.get(), 0, 2 * half, stream_));
    const float4* src = buf.get<float4>();
    float4* dst = reinterpret_cast<float4*>(buf.get<char>() + half);
    const size_t n = half / 16;
    for (int i = 0; i < 3; ++i) RTMB_CUDA(launch_copy_probe(src, dst, n, stream_));
    RTMB_CUDA(cudaEventRecord(ev0_, stream_));
    for (int i = 0; i < iters; ++i) RTMB_CUDA(launch_copy_probe(src, dst, n, stream_));
    RTMB_CUDA(cudaEventRecord(ev1_, stream_));
    RTMB_CUDA(cudaEventSynchronize(ev1_));
    float ms = 0;
    RTMB_CUDA(cudaEventElapsedTime(&ms, ev0_, ev1_));
    *gbps = 2.0 * (double)half * iters / (ms * 1e-3) / 1e9;
    launches_ += iters + 3;
    return RTM_B200_OK;
}

// Post-processing of the finished stack on the device (reference
// src/rtm/imaging.cpp:48-75 applied as at src/main.cpp:211-223).  Plain FP32:
// the running FP32 image with the reference's float operations; otherwise the
// FP64 stack (or the FP64 engine's image), rounded to float at the end.
int Engine::postprocess(float eps_relative, bool compensate_filtered, float* illum_out, float* filtered_out) {
    if (!model_ || !stack_ready_) return fail(RTM_B200_ESTATE, "postprocess before a migration");
    RTMB_CUDA(cudaSetDevice(device_));
    Model& m = *model_;
    const GridDims& g = m.g;
    const size_t n = (size_t)g.nx * g.nz;
    const int row0 = g.nb - g.zs0;
    const bool plain = cfg_.mode == RTM_B200_MODE_PLAIN;
    const bool d64 = !plain || f64_;
    const void* I = plain ? m.img.get() : m.img64.get();
    const void* S = plain ? m.ill.get() : m.ill64.get();
    const size_t es = d64 ? 8 : 4;
    // scratch: max word, dense compensated (or raw) image, float outputs
    const size_t o_dense = 256, o_out = o_dense + ((n * es + 255) & ~(size_t)255);
    RTMB_CUDA(post_.reserve(o_out + 2 * n * 4));
    char* base = post_.get<char>();
    auto* smax = reinterpret_cast<unsigned long long*>(base);
    void* dense = base + o_dense;
    float* out_c = reinterpret_cast<float*>(base + o_out);
    float* out_f = out_c + n;
    RTMB_CUDA(cudaMemsetAsync(smax, 0, sizeof(unsigned long long), stream_));
    RTMB_CUDA(launch_stack_max(S, d64, g.nx, g.nz, g.lds, row0, smax, stream_));
    if (illum_out || (filtered_out && compensate_filtered))
        RTMB_CUDA(launch_compensate(I, S, d64, g.nx, g.nz, g.lds, row0, eps_relative, smax, dense, out_c, stream_));
    if (filtered_out) {
        if (!compensate_filtered) RTMB_CUDA(launch_extract_dense(I, d64, g.nx, g.nz, g.lds, row0, dense, stream_));
        // the reference's weights are float: 1.0f / (dx * dx)
        const float wxf = 1.0f / (m.dx * m.dx), wzf = 1.0f / (m.dz * m.dz);
        const double wx = d64 ? 1.0 / ((double)m.dx * m.dx) : (double)wxf;
        const double wz = d64 ? 1.0 / ((double)m.dz * m.dz) : (double)wzf;
        RTMB_CUDA(launch_laplacian(dense, d64, g.nx, g.nz, wx, wz, out_f, stream_));
    }
    launches_ += 3;
    if (illum_out) RTMB_CUDA(cudaMemcpyAsync(illum_out, out_c, n * 4, cudaMemcpyDefault, stream_));
    if (filtered_out) RTMB_CUDA(cudaMemcpyAsync(filtered_out, out_f, n * 4, cudaMemcpyDefault, stream_));
    RTMB_CUDA(cudaStreamSynchronize(stream_));
    return RTM_B200_OK;
}

int Engine::l2_probe(size_t bytes, int reps, double* gbps) {
    if (!gbps || bytes < 4096 || reps < 1) return fail(RTM_B200_EINVAL, "probe needs >= 4 KiB and >= 1 pass");
    RTMB_CUDA(cudaSetDevice(device_));
    DevMem buf;
    const size_t n = bytes / 16;
    if (buf.alloc(n * 16 + 256) != cudaSuccess) {
        cudaGetLastError();
        return fail(RTM_B200_ENOMEM, "probe buffer");
    }
    RTMB_CUDA(cudaMemsetAsync(buf.get(), 0, n * 16 + 256, stream_));
    const float4* src = buf.get<float4>();
    float* sink = reinterpret_cast<float*>(buf.get<char>() + n * 16);
    for (int i = 0; i < 3; ++i) RTMB_CUDA(launch_l2_read_probe(src, n, reps, -1.0f, sink, stream_));
    RTMB_CUDA(cudaEventRecord(ev0_, stream_));
    constexpr int kLaunches = 5;
    for (int i = 0; i < kLaunches; ++i) RTMB_CUDA(launch_l2_read_probe(src, n, reps, -1.0f, sink, stream_));
    RTMB_CUDA(cudaEventRecord(ev1_, stream_));
    RTMB_CUDA(cudaEventSynchronize(ev1_));
    float ms = 0;
    RTMB_CUDA(cudaEventElapsedTime(&ms, ev0_, ev1_));
    *gbps = (double)n * 16.0 * reps * kLaunches / (ms * 1e-3) / 1e9;
    launches_ += 3 + kLaunches;
    return RTM_B200_OK;
}

int Engine::imaging(const float* fwd, const float* bwd, float* img, float* ill) {
    if (!model_) return fail(RTM_B200_ESTATE, "imaging before setup");
    if (!fwd || !bwd || !img || !ill) return fail(RTM_B200_EINVAL, "null buffer");
    RTMB_CUDA(cudaSetDevice(device_));
    const GridDims& g = model_->g;
    const size_t n = (size_t)g.nx * g.nz, ne = (size_t)g.nxe * g.nze;
    DevMem b;
    RTMB_CUDA(b.alloc((3 * n + ne) * 4));
    float* df = b.get<float>();
    float* di = df + n;
    float* ds = di + n;
    float* de = ds + n;
    RTMB_CUDA(cudaMemcpy(df, fwd, n * 4, cudaMemcpyHostToDevice));
    RTMB_CUDA(cudaMemcpy(di, img, n * 4, cudaMemcpyHostToDevice));
    RTMB_CUDA(cudaMemcpy(ds, ill, n * 4, cudaMemcpyHostToDevice));
    RTMB_CUDA(cudaMemcpy(de, bwd, ne * 4, cudaMemcpyHostToDevice));
    RTMB_CUDA(launch_imaging_dense(df, de, di, ds, g.nx, g.nz, g.nb, g.nze, stream_));
    RTMB_CUDA(cudaStreamSynchronize(stream_));
    RTMB_CUDA(cudaMemcpy(img, di, n * 4, cudaMemcpyDeviceToHost));
    RTMB_CUDA(cudaMemcpy(ill, ds, n * 4, cudaMemcpyDeviceToHost));
    launches_ += 1;
    return RTM_B200_OK;
}

}  // namespace rtmb
