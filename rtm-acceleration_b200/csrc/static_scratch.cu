// static_scratch.cu -- forward modelling of one shot without allocating GPU
// memory (rtm_b200_model_shot_static in include/rtm_b200.h).
//
// Some callers cannot call cudaMalloc: plugins whose host application owns
// every byte of device memory through its own pool and forbids allocations
// behind its back, and latency-critical loops where the implicit device
// synchronisation of cudaMalloc/cudaFree is unacceptable.  The call itself is
// synchronous (plain copies in, the step launches, a wait for its own work).
// For these callers this file keeps all the scratch the step kernel needs -- the two
// wavefield levels, the shot's (v dt)^2, the taper and wavelet tables, the
// receiver lists, the descriptor and the tile list -- in one file-scope device
// array of fixed size.  The array is part of the library's device image: every
// GPU that loads the library holds it until the process exits.
//
// Host code must never use the array's name as a device address: on the host it
// is only a stand-in symbol.  The device address is obtained once per device,
// with that device current, through cudaGetSymbolAddress; the first call on a
// device does that set-up, so that first call should happen before any stream
// capture begins.
//
// Every call shares the array and finds the previous call's contents in it.
// Whatever must start at zero is cleared here or by the kernel itself (the
// first time step writes both wavefield levels in full).  Calls that overlap on
// the GPU would race on the shared array; this function takes a per-device lock
// and waits for its own work before returning, so calls made through it from
// one process never overlap.
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "geometry.hpp"
#include "internal.hpp"
#include "kernels.hpp"
#include "numerics.hpp"
#include "rtm_b200.h"

namespace rtmb {
namespace {

// 32 MiB: a grid of up to ~2.6 million extended cells (e.g. 1400 x 1400 with
// nb = 60) with its receivers and tables.
constexpr size_t kStaticScratchBytes = (size_t)32 << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

std::mutex g_dev_mu[kMaxDevices];
void* g_dev_addr[kMaxDevices] = {};

PFN_cuTensorMapEncodeTiled_v12000 encoder() {
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

size_t up256(size_t b) { return (b + 255) & ~(size_t)255; }

struct Fail {
    int code;
    std::string msg;
};

void set_err(char* err, size_t len, const std::string& m) {
    if (!err || len == 0) return;
    const size_t n = std::min(m.size(), len - 1);
    std::memcpy(err, m.data(), n);
    err[n] = '\0';
}

// Where p lives: 0 host memory (pageable or page-locked), 1 device or managed
// memory of `device`, -1 device memory of another GPU (the step kernel would
// write there without peer access).
int memory_kind(const void* p, int device) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    if (a.type == cudaMemoryTypeManaged) return 1;
    if (a.type == cudaMemoryTypeDevice) return a.device == device ? 1 : -1;
    return 0;
}

#define SS_CUDA(expr)                                                                  \
    do {                                                                               \
        cudaError_t e__ = (expr);                                                      \
        if (e__ != cudaSuccess) throw Fail{RTM_B200_ECUDA, std::string(#expr) + ": " + \
                                                               cudaGetErrorString(e__)}; \
    } while (0)

int model_static(const rtm_b200_static_problem* pr, const rtm_b200_shot* shot, float* traces_out) {
    if (!pr || !shot || !traces_out || !pr->vel) throw Fail{RTM_B200_EINVAL, "null argument"};
    const int half = stencil_half(pr->order);
    if (half < 0) throw Fail{RTM_B200_EINVAL, "unsupported spatial order (use 2, 4, 6, 8, 10 or 12)"};
    if (pr->nb < half + 1) throw Fail{RTM_B200_EINVAL, "--nb must be at least order/2 + 1"};
    if (pr->nx <= 0 || pr->nz <= 0 || pr->nt <= 0 || !(pr->dt > 0.f) || !(pr->dx > 0.f) || !(pr->dz > 0.f))
        throw Fail{RTM_B200_EINVAL, "grid sizes, nt, dt, dx and dz must be positive"};
    if (shot->nrec < 0 || (shot->nrec > 0 && (!shot->rx || !shot->rz)))
        throw Fail{RTM_B200_EINVAL, "receiver arrays are null"};
    const size_t nint = (size_t)pr->nx * pr->nz;
    for (size_t i = 0; i < nint; ++i)
        if (!(pr->vel[i] > 0.0f) || pr->vel[i] > 20000.0f)
            throw Fail{RTM_B200_EINVAL, "velocity model contains a non-physical value"};

    int ndev = 0;
    SS_CUDA(cudaGetDeviceCount(&ndev));
    if (pr->device < 0 || pr->device >= ndev || pr->device >= kMaxDevices)
        throw Fail{RTM_B200_ECUDA, "CUDA device ordinal out of range"};
    SS_CUDA(cudaSetDevice(pr->device));
    std::lock_guard<std::mutex> lock(g_dev_mu[pr->device]);
    if (!g_dev_addr[pr->device]) {
        cudaDeviceProp prop{};
        SS_CUDA(cudaGetDeviceProperties(&prop, pr->device));
        if (prop.major != 10) throw Fail{RTM_B200_ECUDA, "librtm_b200 is built for sm_100a (B200)"};
        void* addr = nullptr;
        SS_CUDA(cudaGetSymbolAddress(&addr, g_static_scratch));
        g_dev_addr[pr->device] = addr;
    }
    char* base = static_cast<char*>(g_dev_addr[pr->device]);
    if (!encoder()) throw Fail{RTM_B200_ECUDA, "cuTensorMapEncodeTiled is unavailable"};

    // ---- host-side tables, exactly as the engine builds them -----------------
    const GridDims g = make_grid(pr->nx, pr->nz, pr->nb, half);
    StepVariant v;
    v.half = half;
    v.tile_x = 16;
    v.warps = 4;
    v.exact = true;
    v.nstage = step_default_stages(v);
    const int TX = step_tile_x(v);
    const int ntx = (g.nxe + TX - 1) / TX;
    const ShotGeometry geo = build_geometry(shot->sx, shot->sz, shot->nrec, shot->rx, shot->rz, g.nx, g.nz, pr->dx,
                                            pr->dz, pr->ox, pr->oz, g.nb);
    std::vector<uint8_t> tflags((size_t)ntx * g.ntz, 0);
    for (int x = 0; x < g.nxe; ++x)
        for (int j = geo.col_start[(size_t)x]; j < geo.col_start[(size_t)x + 1]; ++j)
            tflags[(size_t)(x / TX) * g.ntz + geo.pts[(size_t)j].z / kTileZ] = 1;
    const size_t ntiles = (size_t)ntx * g.ntz;
    const int out_kind = memory_kind(traces_out, pr->device);
    if (out_kind < 0) throw Fail{RTM_B200_EINVAL, "traces_out is device memory of another GPU than problem->device"};
    const bool out_on_device = out_kind == 1;
    const size_t nrec = (size_t)std::max(shot->nrec, 0);

    // ---- carve the static array ---------------------------------------------
    const size_t buf_elems = (size_t)g.nxe * g.ldz;
    size_t off = 0;
    auto take = [&](size_t bytes) { const size_t o = off; off += up256(bytes); return o; };
    const size_t o_fields = take(kFieldBuffers * buf_elems * 4);
    const size_t o_wx = take((size_t)g.nxe * 4);
    const size_t o_wz = take((size_t)g.ldz * 4);
    const size_t o_wav = take((size_t)pr->nt * 4);
    const size_t o_cs = take(geo.col_start.size() * 4);
    const size_t o_pts = take(std::max<size_t>(geo.pts.size(), 1) * sizeof(PointEntry));
    const size_t o_ir = take(std::max<size_t>(geo.ir.size(), 1) * 4);
    const size_t o_desc = take(sizeof(ShotDesc));
    const size_t o_tiles = take(ntiles * sizeof(TileRef));
    const size_t o_ctr = take(sizeof(long long) + sizeof(int));
    const size_t o_rec = take(out_on_device ? 0 : nrec * pr->nt * 4);
    if (off > kStaticScratchBytes)
        throw Fail{RTM_B200_EINVAL, "problem needs " + std::to_string(off) + " bytes of scratch but the static " +
                                        "scratch holds " + std::to_string(kStaticScratchBytes) +
                                        " bytes; use rtm_b200_model_shots instead"};

    std::vector<float> vd(kFieldBuffers * buf_elems, 0.0f);   // levels 0,1 zero; level 2 = (v dt)^2
    const float dt2 = pr->dt * pr->dt;
    float* vdt2 = vd.data() + 2 * buf_elems;
    for (int x = 0; x < g.nxe; ++x) {
        const int ix = std::min(std::max(x - g.nb, 0), g.nx - 1);
        for (int z = 0; z < g.nze; ++z) {
            const int iz = std::min(std::max(z - g.nb, 0), g.nz - 1);
            const float vv = pr->vel[(size_t)ix * g.nz + iz];
            vdt2[(size_t)x * g.ldz + z] = vv * vv * dt2;
        }
    }
    std::vector<float> wx((size_t)g.nxe), wz((size_t)g.ldz, 0.0f);
    for (int i = 0; i < g.nxe; ++i) wx[(size_t)i] = cerjan_taper(i, g.nxe, g.nb, pr->sponge_alpha);
    for (int i = 0; i < g.nze; ++i) wz[(size_t)i] = cerjan_taper(i, g.nze, g.nb, pr->sponge_alpha);
    const std::vector<float> wav = ricker_wavelet(pr->nt, pr->dt, pr->f0);
    const ScaledCoefficients coef = scaled_coefficients(pr->order, pr->dx, pr->dz);

    ShotDesc d{};
    d.nxe = g.nxe; d.nze = g.nze; d.nx = g.nx; d.nz = g.nz; d.nb = g.nb;
    d.model_x0 = 0; d.win_nx = g.nx; d.zs0 = g.zs0; d.lds = g.lds; d.ntz = g.ntz;
    d.nt = pr->nt; d.si = 1; d.nsnap = pr->nt;
    d.g0 = 0; d.total_steps = pr->nt; d.trace_nt = pr->nt;
    d.src_x = geo.src_x; d.src_z = geo.src_z;
    d.flags = kFlagRecord;
    d.snap_type = kSnapF32;
    d.acc_mode = kAccPlain;
    d.field_slot = 0;
    d.nrec = shot->nrec;
    d.c0 = coef.c0;
    for (int k = 0; k <= kMaxHalf; ++k) { d.cx[k] = coef.cx[k]; d.cz[k] = coef.cz[k]; }
    d.ldz_model = g.ldz;
    d.wx = reinterpret_cast<const float*>(base + o_wx);
    d.wz = reinterpret_cast<const float*>(base + o_wz);
    d.wavelet = reinterpret_cast<const float*>(base + o_wav);
    d.col_start = reinterpret_cast<const int*>(base + o_cs);
    d.pts = reinterpret_cast<const PointEntry*>(base + o_pts);
    d.pts_ir = reinterpret_cast<const int*>(base + o_ir);
    d.rec_out = out_on_device ? traces_out : reinterpret_cast<float*>(base + o_rec);

    // ---- upload (copies only; nothing is allocated) ------------------------------
    SS_CUDA(cudaMemcpy(base + o_fields, vd.data(), vd.size() * 4, cudaMemcpyHostToDevice));
    SS_CUDA(cudaMemcpy(base + o_wx, wx.data(), wx.size() * 4, cudaMemcpyHostToDevice));
    SS_CUDA(cudaMemcpy(base + o_wz, wz.data(), wz.size() * 4, cudaMemcpyHostToDevice));
    SS_CUDA(cudaMemcpy(base + o_wav, wav.data(), wav.size() * 4, cudaMemcpyHostToDevice));
    SS_CUDA(cudaMemcpy(base + o_cs, geo.col_start.data(), geo.col_start.size() * 4, cudaMemcpyHostToDevice));
    if (!geo.pts.empty())
        SS_CUDA(cudaMemcpy(base + o_pts, geo.pts.data(), geo.pts.size() * sizeof(PointEntry), cudaMemcpyHostToDevice));
    if (!geo.ir.empty()) SS_CUDA(cudaMemcpy(base + o_ir, geo.ir.data(), geo.ir.size() * 4, cudaMemcpyHostToDevice));
    SS_CUDA(cudaMemcpy(base + o_desc, &d, sizeof(ShotDesc), cudaMemcpyHostToDevice));
    std::vector<TileRef> tiles;
    tiles.reserve(ntiles);
    for (int tz = 0; tz < g.ntz; ++tz)
        for (int tx = 0; tx < ntx; ++tx)
            tiles.push_back(make_tile_ref(d, 0, tx, tz, TX, tflags[(size_t)tx * g.ntz + tz] != 0));
    SS_CUDA(cudaMemcpy(base + o_tiles, tiles.data(), tiles.size() * sizeof(TileRef), cudaMemcpyHostToDevice));
    SS_CUDA(cudaMemset(base + o_ctr, 0, sizeof(long long) + sizeof(int)));   // step counter and error word

    // ---- tensor maps over the three field levels in the static array --------------
    auto encode = [&](bool halo, CUtensorMap* m) {
        const cuuint64_t dims[3] = {(cuuint64_t)g.ldz, (cuuint64_t)g.nxe, (cuuint64_t)kFieldBuffers};
        const cuuint64_t strides[2] = {(cuuint64_t)g.ldz * 4, (cuuint64_t)buf_elems * 4};
        const cuuint32_t box[3] = {(cuuint32_t)(halo ? step_box_z(v) : kTileZ),
                                   (cuuint32_t)(halo ? step_box_x(v) : step_tile_x(v)), 1};
        const cuuint32_t es[3] = {1, 1, 1};
        const CUresult r = encoder()(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base + o_fields, dims, strides, box, es,
                                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) throw Fail{RTM_B200_ECUDA, "cuTensorMapEncodeTiled failed"};
    };
    CUtensorMap map_pc, map_box;
    encode(true, &map_pc);
    encode(false, &map_box);

    // ---- one launch of the step kernel per time step ----------------------------
    StepParams p{};
    p.fields = base + o_fields;
    p.buf_stride = (long long)buf_elems;
    p.slot_stride = (long long)kFieldBuffers * buf_elems;
    p.nbuf = kFieldBuffers;
    p.ldz = g.ldz;
    p.ntiles = (int)ntiles;
    p.descs = reinterpret_cast<const ShotDesc*>(base + o_desc);
    p.tiles = reinterpret_cast<const TileRef*>(base + o_tiles);
    p.stall_tile = -1;
    p.step_counter = reinterpret_cast<const long long*>(base + o_ctr);
    p.error_word = reinterpret_cast<int*>(base + o_ctr + sizeof(long long));
    for (int j = 0; j < pr->nt; ++j) {
        p.step_offset = j;
        SS_CUDA(launch_step(v, map_pc, map_box, p, cudaStreamLegacy));
    }
    SS_CUDA(cudaStreamSynchronize(cudaStreamLegacy));
    int errw = 0;
    SS_CUDA(cudaMemcpy(&errw, base + o_ctr + sizeof(long long), sizeof(int), cudaMemcpyDeviceToHost));
    if (errw) throw Fail{RTM_B200_ETIMEOUT, "a bounded device-side wait gave up"};
    if (!out_on_device)
        SS_CUDA(cudaMemcpy(traces_out, base + o_rec, nrec * pr->nt * 4, cudaMemcpyDeviceToHost));
    return RTM_B200_OK;
}

}  // namespace
}  // namespace rtmb

extern "C" int rtm_b200_model_shot_static(const rtm_b200_static_problem* problem, const rtm_b200_shot* shot,
                                          float* traces_out, char* err, size_t err_len) {
    try {
        const int rc = rtmb::model_static(problem, shot, traces_out);
        rtmb::set_err(err, err_len, "");
        return rc;
    } catch (const rtmb::Fail& f) {
        rtmb::set_err(err, err_len, f.msg);
        return f.code;
    } catch (const std::exception& ex) {
        rtmb::set_err(err, err_len, ex.what());
        return RTM_B200_EINVAL;
    }
}
