// engine.hpp -- the device engine behind the C ABI.
//
// One scheduler serves every mode.  A "job" is one shot in flight; it owns a
// slot (two field buffers in the field pool plus per-shot tables) and a range of
// the snapshot arena.  All jobs advance together, one time step per launch of
// the step kernel, in chunks of C steps captured as one CUDA graph.  Between
// chunks the host retires finished jobs (FP64 stack of their image) and admits
// queued shots into the freed slots and snapshot memory:
//
//   plain  (b200)       : one slot; each shot's imaging adds straight into the
//                         running FP32 image in the reference's order, so the
//                         image is bit-identical to the reference CPU engine;
//   batch  (b200-batch) : as many slots as memory allows; per-shot image and
//                         illumination (Kahan-compensated FP32 by default) are
//                         stacked in FP64 when the shot retires;
//   serve  (b200-serve) : batch scheduling over a queue of requests, each with
//                         its own model, grid, order and time axis, admitted
//                         continuously as slots and snapshot memory free up.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <deque>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "device_util.hpp"
#include "geometry.hpp"
#include "internal.hpp"
#include "numerics.hpp"
#include "rtm_b200.h"

namespace rtmb {

struct StepVariant;   // kernels.hpp

struct ShotData {
    float sx = 0, sz = 0, dt = 0;
    int nrec = 0, nt = 0;
    std::vector<float> rx, rz;
    const float* traces = nullptr;   // borrowed
    int x0 = 0, wnx = 0;              // aperture window (model columns)
};

// One velocity model + time axis + parameters, with its device tables and its
// image accumulators.  setup() makes the engine's own model; every serving
// request makes one.
// Process-wide identity of a Model object, never reused (unlike its address).
inline unsigned long long next_model_uid() {
    static std::atomic<unsigned long long> n{0};
    return ++n;
}

struct Model {
    long long id = 0;
    unsigned long long uid = next_model_uid();
    GridDims g;                        // full model grid
    float dx = 0, dz = 0, ox = 0, oz = 0, dt = 0, f0 = 0, alpha = 0;
    int order = 0, half = 0, nt = 0, si = 1, nsnap = 0;
    ScaledCoefficients coef;
    float vmin = 0, vmax = 0;
    DevMem vdt2, wavelet, wz;
    DevMem img, ill;                   // running image (plain mode), element T
    DevMem img64, ill64;               // FP64 stack (batch/serve)
    std::vector<ShotData> shots;
    size_t next_shot = 0;
    int shots_done = 0;
    // serving bookkeeping
    int state = 0;                     // 0 queued, 1 running, 2 done, -1 failed
    double t_submit = 0, t_start = -1, t_finish = -1;
    std::vector<float> out_img, out_ill;
};

struct Job {
    bool active = false;
    Model* m = nullptr;
    int shot = 0;
    GridDims gs;                       // the shot's own grid (window width)
    int x0 = 0;
    long long g0 = 0;
    int total = 0;                     // steps: nt (modelling) or 2 nt
    int first_phase_step = 0;          // 0, or nt for a backward-only job
    bool modelling = false;
    bool shift_cols = false;           // tiles may start at column H (FMA ring jobs; columns
                                       // [0, H) and [nxe - H, ..) are cleared at set-up)
    float* rec_host = nullptr;
    size_t snap_off = 0, snap_bytes = 0;
    bool owns_snap = false;
    std::vector<std::pair<int, int>> rec_cells;   // (x, z) extended cells holding receivers
    bool tr_wait = false;              // traces still uploading on the copy stream (run_chunk waits
                                       // for them before the job's backward pass)
};

struct Slot {
    DevMem wx, col_start, pts, ir, rec_col, rec_z, traces, rec, acc;
    PinnedMem stage;
    cudaEvent_t staged = nullptr;      // H2D from `stage` finished
    cudaEvent_t free_ev = nullptr;     // step stream: work queued before a new job's trace upload
    cudaEvent_t tr_ready = nullptr;    // copy stream: the job's traces have landed
};

class Engine {
public:
    explicit Engine(const rtm_b200_config& cfg);
    ~Engine();
    int init();

    int setup(const float* vel, int nx, int nz, float dx, float dz, float ox, float oz, int nt, float dt);
    int migrate(const rtm_b200_shot* shots, int nshots, float* img, float* ill, double* img64, double* ill64);
    int model_shots(const rtm_b200_shot* shots, int nshots, float* out);
    int forward(const rtm_b200_shot* shot, float* snaps, float* rec);
    int backward(const rtm_b200_shot* shot, const float* snaps, float* img, float* ill);
    int imaging(const float* fwd, const float* bwd, float* img, float* ill);
    int postprocess(float eps_relative, bool compensate_filtered, float* illum_out, float* filtered_out);

    int submit(const rtm_b200_request* req, long long* ticket);
    int serve_step(int max_steps, int* pending);
    int poll(long long ticket, rtm_b200_request_status* st, float* img, float* ill);
    int drain();

    int memory_probe(size_t bytes, int iters, double* gbps);
    int l2_probe(size_t bytes, int reps, double* gbps);
    double clock() const;
    int num_snapshots() const { return model_ ? model_->nsnap : 0; }
    long long snapshot_bytes() const;
    const std::string& last_error() const { return error_; }
    const std::string& device_name() const { return device_name_; }
    rtm_b200_times times{};

    int fail(int code, std::string msg) {
        error_ = std::move(msg);
        return code;
    }

private:
    // set-up helpers
    int validate_params(int nx, int nz, float dx, float dz, int order, int nb, int si, int nt, float dt,
                        float f0, const float* vel, float* vmin, float* vmax);
    int build_model(Model& m, const float* vel, int nx, int nz, float dx, float dz, float ox, float oz,
                    int order, int nt, float dt, int si, float f0);
    int copy_shots(Model& m, const rtm_b200_shot* shots, int nshots, bool need_traces);
    size_t elem() const { return f64_ ? 8 : 4; }
    int snap_type() const;
    size_t snap_alloc_bytes(const Model& m, const GridDims& gs) const;

    // pool / slots
    int ensure_pool(int nslots, int nxe_cap, int ldz_cap);
    int ensure_slot(int s, const Model& m, const ShotData& sh, const GridDims& gs, bool modelling);
    int encode_map(int half, bool with_halo, CUtensorMap* out);
    StepVariant variant(int half) const;   // step-kernel variant for a stencil half-order

    // scheduling
    int start_job(int slot, Model* m, int shot, bool modelling, float* rec_host, int backward_only,
                  size_t snap_off, size_t snap_bytes, bool owns_snap);
    int retire_finished();
    int finish_job(int slot);
    int run_chunk(int steps);
    int build_tiles();
    int check_device_error();
    void abort_jobs();
    int run_queue(std::deque<std::pair<Model*, int>>& q, bool modelling, float* rec_base,
                  const std::vector<size_t>* rec_offsets);
    int admit_from(std::deque<std::pair<Model*, int>>& q, bool modelling, float* rec_base,
                   const std::vector<size_t>* rec_offsets, int* admitted, int limit = -1);
    int active_jobs() const;
    int chunk_for(const Model& m) const;
    int zero_model_images(Model& m);
    int finalize_model_image(Model& m, float* img, float* ill, double* img64, double* ill64);

    // serving
    int serve_admit();
    int serve_finish_models();

    rtm_b200_config cfg_{};
    bool f64_ = false;
    bool auto_arith_ = false;                // arithmetic AUTO: modelling runs IEEE
    bool recon_ = false;                     // snapshot-free source reconstruction
    int nbuf_ = kFieldBuffers;               // field buffers per slot
    bool modelling_now_ = false;             // inside model_shots
    bool exact() const {
        return cfg_.arithmetic == RTM_B200_ARITH_IEEE || (auto_arith_ && modelling_now_);
    }
    bool inited_ = false;
    int device_ = 0;
    std::string error_;
    std::string device_name_;
    cudaStream_t stream_ = nullptr;
    cudaStream_t copy_stream_ = nullptr;   // trace uploads that overlap the forward pass
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
    std::chrono::steady_clock::time_point t0_;

    std::unique_ptr<Model> model_;           // the setup() model
    bool stack_ready_ = false;               // model_'s stack holds a finished migration
    DevMem post_;                            // post-processing scratch

    // field pool: T[nslots][nbuf][nxe_cap][ldz_cap], then (FP32) one more
    // buffer holding a model's (v dt)^2 table, which interior tiles of every shot
    // on that model load instead of their slot's copy, so that it stays in L2
    DevMem pool_;
    int nslots_ = 0, nxe_cap_ = 0, ldz_cap_ = 0;
    unsigned long long shared_vd_uid_ = 0;   // model whose table the shared buffer holds (0: none)
    int shared_vd_buf() const { return nslots_ * nbuf_; }
    int pool_buffers() const { return nslots_ * nbuf_ + (f64_ ? 0 : 1); }
    int share_model_vdt2(const Model* m);
    bool shifted_bands() const;   // an active job's bands start at a row other than 0
    bool band_shift_ = true;      // FMA ring jobs may start their bands at row H & ~3
    struct MapPair { CUtensorMap pc, box; };
    std::map<int, MapPair> maps_;            // by (half, tile width): p^n box with halo; 128 x TX box
    std::vector<Slot> slots_;
    std::vector<Job> jobs_;
    DevMem descs_;                           // ShotDesc[nslots]
    std::vector<ShotDesc> host_descs_;
    DevMem counter_;                         // long long global step
    long long g_ = 0;                        // host mirror of the counter
    DevMem errword_;

    // snapshot arena
    DevMem arena_;
    RangeAllocator alloc_;
    size_t arena_bytes_ = 0;

    // tiles and the captured chunk graph
    DevMem tiles_;
    struct Group { int half; int offset; int count; };
    std::vector<Group> groups_;
    std::vector<long long> tile_sig_;
    bool tiles_dirty_ = true;
    cudaGraphExec_t graph_ = nullptr;
    std::vector<long long> graph_sig_;
    int graph_steps_ = 0;
    int launches_ = 0;
    int tile_x_ = 16;                        // ring kernel: tile width (16 or 32 columns)
    int warps_ = 4;                          // ring kernel: consumer warps per CTA
    int spare_ = 0;                          // ring kernel: leave one CTA slot per SM free
    int stage_override_ = 0;                 // ring kernel: pipeline stages (0 = default)
    int stall_tile_ = -1;                    // failure-detection test hook (RTM_B200_STALL_TILE)
    // Autotuner: the fastest step kernel and parameters measured on real steps,
    // cached per job mix (stencil orders, tile rows, shots in flight).
    bool autotune_ = false;
    int kind_ = 0;                           // kStepRing or kStepMarch (autotuned)
    int march_m_ = 3;                        // march strip length, units of 2H+1 columns
    int pin_kind_ = -1;                      // step kernel pinned by RTM_B200_STEP_KERNEL (-1: tuned)
public:
    struct TuneChoice { int kind, warps, tile_x, stages, march_m, spare; };
private:
    std::map<std::vector<long long>, TuneChoice> tuned_;
    std::vector<long long> tune_key() const;
    int run_steps(int steps);
    cudaEvent_t tune_ev0_ = nullptr, tune_ev1_ = nullptr;
public:
    struct TuneRecord {
        std::vector<long long> key;
        TuneChoice pick;
        std::vector<TuneChoice> cands;
        std::vector<double> us_per_step;
    };
    std::vector<TuneRecord> tune_log_;
    // Shots in flight of the batch engine, tuned across migrate calls on the
    // same survey: each early call runs one candidate on real work.
    struct InflightTune {
        std::vector<long long> key;          // grid, order, nt, snapshot type, shots
        std::vector<int> cands;
        std::vector<double> shots_per_s;     // measured (device time), 0 = untested
        int pick = 0;                        // 0 until every candidate ran
    };
    std::vector<InflightTune> inflight_log_;
private:
    // backpressure: at most kChunksInFlight chunks queued ahead of the GPU
    static constexpr int kChunksInFlight = 3;
    cudaEvent_t chunk_ev_[kChunksInFlight] = {};
    long long chunk_k_ = 0;

    // backward-only support: device snapshots kept from the last forward()
    size_t keep_snap_off_ = 0, keep_snap_bytes_ = 0;
    bool keep_snap_ = false;

    // serving
    std::map<long long, std::unique_ptr<Model>> requests_;
    std::deque<long long> req_queue_;
    long long next_ticket_ = 1;
    std::deque<std::pair<Model*, int>> serve_q_;
    bool serve_ready_ = false;
    int serve_init(const Model& first);
    struct Finishing {
        long long ticket;
        cudaEvent_t ev;
        PinnedMem host;
    };
    std::vector<std::unique_ptr<Finishing>> finishing_;
    int serve_collect(bool wait);
};

}  // namespace rtmb
