// rtm_b200_engine.hpp -- C++17 host API of the B200 RTM engine.
//
// The same engine interface as the reference project (Marouane-Djabri/
// RTM-Acceleration): the RTMEngine virtuals of include/rtm_engine.hpp:20-83,
// make_engine / list_engines of include/rtm_factory.hpp:19-23, the value types
// of include/rtm_types.hpp:10-65 and the readers of include/rtm_io.hpp:9-37,
// kept in namespace rtm_b200 so a program can link both.  B200RTM implements
// the interface over the C ABI of librtm_b200.so (rtm_b200.h) and throws
// std::runtime_error on a non-zero status, like the reference engines.
#pragma once

#include <cstddef>
#include <memory>
#include <string>
#include <vector>

#include "rtm_b200.h"

namespace rtm_b200 {

// Interior grid plus the sponge width; arrays are zfast: v[ix*nz + iz].
struct Grid {
    int nx = 0, nz = 0, nb = 0;
    float dx = 10.0f, dz = 10.0f, ox = 0.0f, oz = 0.0f;
    int nxe() const { return nx + 2 * nb; }
    int nze() const { return nz + 2 * nb; }
    std::size_t n_interior() const { return (std::size_t)nx * nz; }
    std::size_t n_extended() const { return (std::size_t)nxe() * nze(); }
};

struct TimeAxis {
    int nt = 0;
    float dt = 0.0f;
};

// The reference's RTMParams defaults.
struct RTMParams {
    int nb = 60;
    int order = 8;
    float sponge_alpha = 0.0053f;
    int store_interval = 1;
    float f0 = 12.0f;
    bool verbose = true;
};

struct VelocityModel {
    Grid grid;
    std::vector<float> v;   // nx*nz, zfast, m/s
    float vmin() const;
    float vmax() const;
};

// One shot gather; traces are trace-major: traces[ir*nt + it].
struct ShotRecord {
    float sx = 0.0f, sz = 0.0f;
    std::vector<float> rx, rz;
    int nt = 0;
    float dt = 0.0f;
    std::vector<float> traces;
    int window_x0 = 0, window_nx = 0;   // aperture window in model columns (0,0: whole model)
    int nrec() const { return (int)rx.size(); }
};

struct StageTimes {
    double io = 0, forward = 0, backward = 0, imaging = 0, total = 0;
    double h2d = 0, kernel = 0, d2h = 0;
    void reset() { *this = StageTimes(); }
};

// The engine interface (same members as the reference's RTMEngine).
class RTMEngine {
public:
    virtual ~RTMEngine() = default;
    virtual const char* name() const = 0;
    virtual void setup(const VelocityModel& model, const RTMParams& par, const TimeAxis& ta) = 0;
    virtual void forward_propagation(const ShotRecord& shot, std::vector<float>* snapshots,
                                     std::vector<float>* recorded) = 0;
    virtual void backward_propagation(const ShotRecord& shot, const std::vector<float>& snapshots,
                                      std::vector<float>& image, std::vector<float>& illumination) = 0;
    virtual void imaging(const float* fwd_snapshot, const float* bwd_extended, std::vector<float>& image,
                         std::vector<float>& illumination) = 0;
    virtual void migrate(const std::vector<ShotRecord>& shots, std::vector<float>& image,
                         std::vector<float>& illumination) = 0;
    virtual void model_shot(ShotRecord& shot) = 0;

    const Grid& grid() const { return g_; }
    const RTMParams& params() const { return par_; }
    const TimeAxis& time_axis() const { return ta_; }
    int num_snapshots() const { return nsnap_; }
    std::size_t snapshot_bytes() const { return (std::size_t)nsnap_ * g_.n_interior() * sizeof(float); }
    virtual int num_threads() const { return 1; }
    virtual int num_devices() const { return 0; }
    virtual std::string device_name() const { return "cpu"; }
    virtual bool is_gpu() const { return false; }

    StageTimes times;

protected:
    Grid g_;
    RTMParams par_;
    TimeAxis ta_;
    int nsnap_ = 0;
};

// Engine options beyond the reference's RTMParams.
struct B200Options {
    int mode = RTM_B200_MODE_PLAIN;
    int device = 0;
    int snap_precision = RTM_B200_SNAP_F32;
    int arithmetic = RTM_B200_ARITH_AUTO;
    int accumulation = RTM_B200_ACC_COMPENSATED;
    int max_shots_in_flight = 0;
    int tile_cols = 0;
};

// The B200 engine over librtm_b200.so (engines b200, b200-batch, b200-serve).
class B200RTM : public RTMEngine {
public:
    explicit B200RTM(const B200Options& opt);
    ~B200RTM() override;
    B200RTM(const B200RTM&) = delete;
    B200RTM& operator=(const B200RTM&) = delete;

    const char* name() const override;
    void setup(const VelocityModel& model, const RTMParams& par, const TimeAxis& ta) override;
    void forward_propagation(const ShotRecord& shot, std::vector<float>* snapshots,
                             std::vector<float>* recorded) override;
    void backward_propagation(const ShotRecord& shot, const std::vector<float>& snapshots,
                              std::vector<float>& image, std::vector<float>& illumination) override;
    void imaging(const float* fwd_snapshot, const float* bwd_extended, std::vector<float>& image,
                 std::vector<float>& illumination) override;
    void migrate(const std::vector<ShotRecord>& shots, std::vector<float>& image,
                 std::vector<float>& illumination) override;
    void model_shot(ShotRecord& shot) override;
    // All shots modelled in one call (batched on the device).
    void model_shots(std::vector<ShotRecord>& shots);
    // The `_illum` and `_filtered` outputs of the last migrate(), computed on
    // the device (rtm_b200_postprocess); either pointer may be null.
    void postprocess(float eps_relative, bool compensate_filtered, std::vector<float>* illum_out,
                     std::vector<float>* filtered_out);

    int num_devices() const override { return 1; }
    std::string device_name() const override;
    bool is_gpu() const override { return true; }
    rtm_b200_times raw_times() const;

private:
    void check(int rc, const char* what) const;
    void copy_times();
    B200Options opt_;
    rtm_b200_engine* h_ = nullptr;
};

// Factory (reference make_engine / list_engines).  Unknown names throw.
std::unique_ptr<RTMEngine> make_engine(const std::string& engine_name, int requested_gpus = 1,
                                       const B200Options* options = nullptr);
std::vector<std::string> list_engines();

// Shared numerics (host; the C ABI's implementation).
std::vector<float> stencil_coefficients(int order);
float ricker(float t, float f0);
float max_stable_dt(float vmax, const Grid& g, int order);
float points_per_wavelength(float vmin, float f0, const Grid& g);
void mute_direct_wave(ShotRecord& s, float v_surface, float t_pad, float t_taper);

// Post-processing of a finished stack (separate outputs only).
void illumination_compensation(std::vector<float>& image, const std::vector<float>& illumination,
                               float eps_relative);
void laplacian_filter(std::vector<float>& image, const Grid& g);

// Image comparison in double precision, and the reference's default gate.
struct ImageDiff {
    std::size_t n = 0;
    double max_abs = 0, mean_abs = 0, rms = 0, l2_relative = 0, max_relative = 0, correlation = 0;
    double ref_max_abs = 0, test_max_abs = 0;
    std::size_t argmax = 0;
};
ImageDiff compare_images(const std::vector<float>& ref, const std::vector<float>& test);
bool gate_pass(const ImageDiff& d, double l2_max = 1e-5, double corr_min = 0.9999);

namespace io {
struct VelocityHeader {
    int nx = 0, nz = 0;
    float dx = 10.0f, dz = 10.0f, ox = 0.0f, oz = 0.0f;
    std::string layout = "zfast";
};
bool read_header_file(const std::string& path, VelocityHeader& h);
void write_header_file(const std::string& path, const VelocityHeader& h);
VelocityModel read_velocity_raw(const std::string& path, const VelocityHeader& h);
void write_velocity_raw(const std::string& path, const VelocityModel& m);
std::vector<ShotRecord> read_shots_raw(const std::string& path);
std::vector<ShotRecord> read_shots_segy(const std::string& path, float src_depth, float rec_depth);
std::vector<ShotRecord> read_shots(const std::string& path, float src_depth = 10.0f, float rec_depth = 10.0f);
void write_shots_raw(const std::string& path, const std::vector<ShotRecord>& shots);
void write_raw_floats(const std::string& path, const std::vector<float>& v);
std::vector<float> read_raw_floats(const std::string& path);
}  // namespace io

}  // namespace rtm_b200
