// kernels.hpp -- host-callable launchers for librtm_b200's device code.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include "internal.hpp"
#include "march_kernel.cuh"
#include "step_kernel.cuh"

namespace rtmb {

// Compile-time variant of the step kernel, chosen at run time.
struct StepVariant {
    bool f64 = false;   // double fields (the FP64 run)
    int half = 4;       // order / 2
    bool exact = true;  // IEEE unfused float arithmetic (bit-identical path)
    int tile_x = 16;    // ring kernel: tile of 128 rows x tile_x (16 or 32) columns
    int warps = 8;      // ring kernel: consumer warps per CTA (see step_shape_supported)
    bool spare = false; // ring kernel: grid leaves one CTA slot per SM free (shapes of 2+ CTAs/SM)
    int nstage = 3;     // shared-memory pipeline stages, 2..kMaxStages
    int kind = 0;       // 0: TMA ring kernel (step_kernel); 1: register march (march_kernel, FP32)
    int march_m = 3;    // march: strip length in units of 2*half+1 columns (1..9)
};

constexpr int kStepRing = 0;
constexpr int kStepMarch = 1;

// Ring-kernel shapes (consumer warps x tile width) and the CTAs per SM each is
// built for.  An SM's registers are split over its four sub-partitions and
// warps are dealt to them round-robin, so the per-thread register budget
// follows the most loaded sub-partition:
//   FP32  4 warps x 16 columns, 3 CTAs/SM (15 warps: 128 registers), 2 column
//         pairs per warp per tile;
//   FP32  8 warps x 16 columns, 2 CTAs/SM (18 warps:  96 registers), 1 pair;
//   FP32  8 warps x 32 columns, 1 CTA/SM  ( 9 warps: 168 registers), 2 pairs;
//   FP64  8 warps x 16 or 32 columns, 1 CTA/SM.
inline bool step_shape_supported(bool f64, int warps, int tile_x) {
    if (f64) return warps == 8 && (tile_x == 16 || tile_x == 32);
    return (warps == 4 && tile_x == 16) || (warps == 8 && (tile_x == 16 || tile_x == 32));
}
template <typename T, int NCW, int TX>
constexpr int step_ctas_per_sm() { return sizeof(T) == 8 ? 1 : (NCW == 4 ? 3 : (TX == 16 ? 2 : 1)); }
inline int step_ctas_per_sm(const StepVariant& v) {
    return v.f64 ? 1 : (v.warps == 4 ? 3 : (v.tile_x == 16 ? 2 : 1));
}
inline int step_threads(const StepVariant& v) { return (v.warps + 1) * 32; }

inline int step_tile_x(const StepVariant& v) {
    return v.kind == kStepMarch ? (2 * v.half + 1) * v.march_m : v.tile_x;
}
inline int step_halo_rows(const StepVariant& v) { return (v.half + 3) & ~3; }
inline int step_box_z(const StepVariant& v) { return kTileZ + 2 * step_halo_rows(v); }
inline int step_box_x(const StepVariant& v) { return step_tile_x(v) + 2 * v.half; }
int step_stage_bytes(const StepVariant& v);
int step_smem_bytes(const StepVariant& v);
bool step_variant_supported(const StepVariant& v);
// Deepest pipeline that keeps the variant's CTAs per SM (step_ctas_per_sm)
// inside the SM's shared memory.
int step_default_stages(const StepVariant& v);

// Sets the kernel's shared-memory attribute (call before any stream capture).
cudaError_t prepare_step(const StepVariant& v);

// Resident CTAs of the persistent step kernel on this device (grid cap).
int step_max_grid(const StepVariant& v);

// Launch one time step over p.ntiles tiles (grid = min(ntiles, resident CTAs)),
// as a programmatic dependent launch: its CTAs may start while the previous
// kernel in the stream drains and wait in-kernel for it to finish.
// map_pc: box of p^n with halo (step_box_z x step_box_x); map_box: box of
// 128 x step_tile_x (p^{n-1} and (v dt)^2).  Both describe the field pool.
cudaError_t launch_step(const StepVariant& v, const CUtensorMap& map_pc, const CUtensorMap& map_box,
                        const StepParams& p, cudaStream_t s);

// Fill a slot's (v dt)^2 buffer (nxe columns x ldz rows) from the model table,
// columns clamped to the aperture window [x0, x0+win_nx).
cudaError_t launch_slot_vdt2(void* dst, bool f64, int ldz, int nxe, const float* model, int ldz_model, int nb,
                             int win_nx, int x0, cudaStream_t s);

cudaError_t launch_advance_counter(long long* counter, int by, cudaStream_t s);

// dst[ix*nz+iz] = src[ix*lds + row0 + iz]   (padded image/snapshot -> dense)
cudaError_t launch_extract_f32(const float* src, int lds, int row0, float* dst, int nx, int nz, int count,
                               cudaStream_t s);
cudaError_t launch_extract_f64_to_f32(const double* src, int lds, int row0, float* dst, int nx, int nz,
                                      cudaStream_t s);
cudaError_t launch_extract_f64(const double* src, int lds, int row0, double* dst, int nx, int nz, cudaStream_t s);
// dense -> padded for `count` consecutive snapshots (host snapshots uploaded for backward)
cudaError_t launch_insert_f32(const float* src, int nx, int nz, float* dst, int lds, int row0, int count,
                              cudaStream_t s);
cudaError_t launch_insert_f64(const double* src, int nx, int nz, double* dst, int lds, int row0, int count,
                              cudaStream_t s);

// FP64 cross-shot stack of one shot's image/illumination, shot columns placed
// at model column `col0`.  Ic / Sc are the Kahan compensation words (BF16 bit
// patterns); they may be null (uncompensated sums).
cudaError_t launch_stack_f32(const float* I, const uint16_t* Ic, const float* S, const uint16_t* Sc, double* I64,
                             double* S64, int nx, int lds, int col0, cudaStream_t s);
cudaError_t launch_stack_f64(const double* I, const double* S, double* I64, double* S64, int nx, int lds,
                             int col0, cudaStream_t s);

// One zero-lag imaging step on dense arrays (reference imaging.cpp:25-40).
cudaError_t launch_imaging_dense(const float* fwd, const float* bwd_ext, float* I, float* S, int nx, int nz,
                                 int nb, int nze, cudaStream_t s);

// dst[i] = src[i] over n float4 elements (bandwidth probe).
cudaError_t launch_copy_probe(const float4* src, float4* dst, size_t n, cudaStream_t s);

// Post-processing of a finished stack (reference illumination_compensation and
// laplacian_filter, src/rtm/imaging.cpp:48-75).  S and I are in the padded
// stack layout (nx columns of lds rows, interior rows from row0).
// smax_bits <- bits of max(0, max S) as a double (S >= 0, so the bit patterns
// order like the values); clear it to 0 first.
cudaError_t launch_stack_max(const void* S, bool f64, int nx, int nz, int lds, int row0,
                             unsigned long long* smax_bits, cudaStream_t s);
// dense[ix*nz+iz] = I / (S + eps), eps = eps_rel * smax + 1e-30, in the
// stack's precision (FP32: the reference's float operations bit for bit).
// dense is T (float or double); out (may be null) receives it as float.
cudaError_t launch_compensate(const void* I, const void* S, bool f64, int nx, int nz, int lds, int row0,
                              float eps_rel, const unsigned long long* smax_bits, void* dense, float* out,
                              cudaStream_t s);
// dense (nx*nz, T) -> raw image copy (no compensation), for the filter input.
cudaError_t launch_extract_dense(const void* I, bool f64, int nx, int nz, int lds, int row0, void* dense,
                                 cudaStream_t s);
// out[i] = wx (in[i+nz] - 2 in[i] + in[i-nz]) + wz (in[i+1] - 2 in[i] + in[i-1])
// on the interior, 0 on the outermost rows and columns; FP32 in the reference's
// operation order, or FP64 for a double input.
cudaError_t launch_laplacian(const void* in, bool f64, int nx, int nz, double wx, double wz, float* out,
                             cudaStream_t s);

// Reads n float4 elements `reps` times in one launch, through L2 (no L1), and
// folds them into a sum nothing uses unless it equals `never`: the L2 read
// bandwidth of a buffer small enough to stay resident.
cudaError_t launch_l2_read_probe(const float4* src, size_t n, int reps, float never, float* sink, cudaStream_t s);

// float -> double widening of a dense array.
cudaError_t launch_widen(const float* src, double* dst, size_t n, cudaStream_t s);

}  // namespace rtmb
