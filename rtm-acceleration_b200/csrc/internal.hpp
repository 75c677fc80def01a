// internal.hpp -- data structures shared by the host engine and the sm_100a
// kernels of librtm_b200.  Not part of the public ABI.
//
// Device layout (every array is "zfast", depth contiguous, like the reference's
// index = ix*nz + iz, include/rtm_types.hpp:10-15 of the reference):
//
//   field pool   T[nslot][3][NXE][LDZ]  per shot slot: two time levels (the
//                leapfrog runs in place: p^{n+1} overwrites p^{n-1}) and the
//                shot's (v dt)^2 on its extended grid; a shot's extended grid
//                (nxe x nze) sits in the top-left corner of its slot.  LDZ is a
//                multiple of 8 so every column starts on a 32-byte boundary.
//   vdt2 model   float[model_nx][LDZ]  (v dt)^2 for every interior model column,
//                extended in depth by edge replication; a shot's slot copy is
//                extended in x by clamping to its aperture window, which gives
//                each window its own edge replication (reference
//                src/rtm/rtm_cpu.cpp:33-42 on the cropped model).
//   snapshots    S[nsnap][nx][lds]  interior columns, rows [zs0, zs0+lds) of the
//                extended grid (zs0 = nb rounded down to 4, lds multiple of 4).
//   image/illum  A[nx][lds]          same layout as one snapshot.
#pragma once
#include <cstdint>
#include <cstddef>

namespace rtmb {

constexpr int kMaxHalf = 6;
constexpr int kTileZ = 128;          // rows per tile: 32 lanes x 4 consecutive rows

enum SnapType : int { kSnapF32 = 0, kSnapBF16 = 1, kSnapF16 = 2, kSnapF64 = 3 };
enum AccMode : int {
    kAccPlain = 0,        // I += f*b straight into the shared image (reference order)
    kAccCompensated = 1,  // per-shot Kahan-compensated sums (sum, comp) pairs
};
enum ShotFlags : int {
    kFlagSnapshots = 1,   // forward pass stores snapshots
    kFlagImage = 2,       // backward pass runs (and images)
    kFlagRecord = 4,      // forward pass records traces at the receivers
};

// One receiver cell of a shot: extended depth index and the receivers
// (in ascending ir order) that sit on it.
struct PointEntry {
    int z;          // extended depth index of the cell
    int ir_begin;   // first entry in the shot's receiver index list
    int ir_count;   // number of receivers on this cell
    int pad;
};

// Per shot slot; lives in device memory, read by every CTA of that shot.
struct ShotDesc {
    // grid
    int nxe, nze, nx, nz, nb;
    int model_x0;        // first model column of this shot's aperture window
    int win_nx;          // window width in model columns (== nx)
    int zs0, lds;        // snapshot/image row origin (extended z) and pitch
    int ntz;             // tiles in z (scale-exponent stride)
    int ntx;             // tiles in x
    // time
    int nt, si, nsnap;
    long long g0;        // global step at which forward step 0 runs
    int total_steps;     // nt (modelling) or 2*nt (migration)
    int trace_nt;        // stride of the trace array (samples per trace)
    int src_x, src_z;    // extended coordinates of the source cell
    int flags;
    int snap_type;
    int acc_mode;
    int field_slot;
    int nrec;
    // stencil coefficients (float, widened in double kernels)
    float c0, cx[kMaxHalf + 1], cz[kMaxHalf + 1];
    // pointers
    const float* vdt2;       // model table [model_nx][ldz_model]
    int ldz_model;
    int pad0;
    const float* wx;         // nxe taper weights
    const float* wz;         // ldz taper weights (zero past nze)
    const float* wavelet;    // nt
    const float* traces;     // nrec * trace_nt, trace-major
    const int* col_start;    // nxe+1 offsets into pts
    const uint8_t* tile_pts; // ntx*ntz flags: tile holds receiver cells
    const PointEntry* pts;
    const int* pts_ir;
    float* rec_out;          // nrec * nt trace-major (modelling)
    void* snap;              // nsnap * nx * lds  (snap_type)
    int8_t* snap_exp;        // nsnap * nx * ntz  power-of-two scale exponents
    void* img;               // nx * lds  (float, or double for T=double)
    void* ill;
    void* img_c;             // compensation words (kAccCompensated)
    void* ill_c;
};

constexpr int kFieldBuffers = 3;     // p^n / p^{n+1}, p^{n-1}, (v dt)^2

// One CTA's work item.
struct TileRef {
    int slot;        // index into the descriptor array
    int tx, tz;      // tile coordinates inside the shot's extended grid
    int pad;
};

// Error bits written by the kernels into the engine's device error word.
enum DeviceError : int {
    kErrTmaTimeout = 1,
    kErrBadTile = 2,
    kErrBarrierTimeout = 4,
};

}  // namespace rtmb
