// internal.hpp -- data structures shared by the host engine and the sm_100a
// kernels of librtm_b200.  Not part of the public ABI.
//
// Device layout (every array is "zfast", depth contiguous, like the reference's
// index = ix*nz + iz, include/rtm_types.hpp:10-15 of the reference):
//
//   field pool   T[nslot][nbuf][NXE][LDZ]  per shot slot: two time levels (the
//                leapfrog runs in place: p^{n+1} overwrites p^{n-1}) and the
//                shot's (v dt)^2 on its extended grid; with source
//                reconstruction two more levels (nbuf = 5) hold the receiver
//                field of the backward pass while the first two hold the source
//                field running backwards.  A shot's extended grid (nxe x nze)
//                sits in the top-left corner of its slot.  LDZ is a multiple of
//                8 so every column starts on a 32-byte boundary.
//   vdt2 model   float[model_nx][LDZ]  (v dt)^2 for every interior model column,
//                extended in depth by edge replication; a shot's slot copy is
//                extended in x by clamping to its aperture window, which gives
//                each window its own edge replication (reference
//                src/rtm/rtm_cpu.cpp:33-42 on the cropped model).
//   snapshots    S[nsnap][nx][lds]  interior columns, rows [zs0, zs0+lds) of the
//                extended grid (zs0 = nb rounded down to 4, lds multiple of 4).
//   boundary     B[nt-1][bsize]  source reconstruction instead of snapshots:
//   strips       level m = 1..nt-1 of the source field on the band of H cells
//                around the interior (left, right: H x nz; top, bottom: nx x H).
//   image/illum  A[nx][lds]          same layout as one snapshot.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cstring>

namespace rtmb {

constexpr int kMaxHalf = 6;
constexpr int kCoefSlots = 8;   // cx / cz entries in ShotDesc: kMaxHalf + 1, rounded up to a float4 pair
constexpr int kTileZ = 128;          // rows per tile: 32 lanes x 4 consecutive rows

enum SnapType : int { kSnapF32 = 0, kSnapBF16 = 1, kSnapF16 = 2, kSnapF64 = 3, kSnapNone = 4 };
enum AccMode : int {
    kAccPlain = 0,        // I += f*b straight into the shared image (reference order)
    kAccCompensated = 1,  // per-shot Kahan-compensated sums (sum, comp) pairs
};
enum ShotFlags : int {
    kFlagSnapshots = 1,   // forward pass stores snapshots
    kFlagImage = 2,       // backward pass runs (and images)
    kFlagRecord = 4,      // forward pass records traces at the receivers
    kFlagRecon = 8,       // no snapshots: the forward pass stores the boundary
                          // strips, the backward pass rebuilds the source field
    kFlagSourceTile = 64, // TileRef only: a tile of the source field running
                          // backwards (reconstruction), not of the shot's field
    kFlagBandTile = 128,  // TileRef only: the tile holds cells of the boundary
                          // strip band (reconstruction)
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
    int ntz;             // 128-row bands (stride of the snapshot scale exponents)
    int bsize;           // reconstruction: boundary-strip cells per level
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
    // stencil coefficients (float, widened in double kernels); cx and cz start
    // on 16-byte boundaries so the step kernel reads them as float4 pairs
    float c0;
    alignas(16) float cx[kCoefSlots];
    alignas(16) float cz[kCoefSlots];
    // pointers
    const float* vdt2;       // model table [model_nx][ldz_model]
    int ldz_model;
    int pad0;
    const float* wx;         // nxe taper weights
    const float* wz;         // ldz taper weights (zero past nze)
    const float* wavelet;    // nt
    const float* traces;     // nrec * trace_nt, trace-major
    const int* col_start;    // nxe+1 offsets into pts
    const PointEntry* pts;
    const int* pts_ir;
    const int* rec_col;      // nxe+1 receiver offsets per column (null: not staged)
    const int* rec_zs;       // extended row of each receiver, pts_ir order
    float* rec_out;          // nrec * nt trace-major (modelling)
    void* snap;              // nsnap * nx * lds  (snap_type)
    int8_t* snap_exp;        // nsnap * nx * ntz  power-of-two scale exponents
    void* img;               // nx * lds  (float, or double for T=double)
    void* ill;
    void* img_c;             // Kahan compensation words, BF16 (kAccCompensated)
    void* ill_c;
};

constexpr int kFieldBuffers = 3;     // p^n / p^{n+1}, p^{n-1}, (v dt)^2
constexpr int kReconBuffers = 5;     // + the receiver field's two levels

// Index of extended cell (x, z) in a boundary strip level, or -1 when the cell
// is not in the band of H cells around the interior [nb, nb+nx) x [nb, nb+nz).
#if defined(__CUDACC__)
#define RTMB_HOST_DEVICE __host__ __device__
#else
#define RTMB_HOST_DEVICE
#endif
RTMB_HOST_DEVICE inline int strip_index(int x, int z, int nb, int nx, int nz, int H) {
    const bool zin = z >= nb && z < nb + nz, xin = x >= nb && x < nb + nx;
    if (zin && x >= nb - H && x < nb) return (x - (nb - H)) * nz + (z - nb);
    if (zin && x >= nb + nx && x < nb + nx + H) return (H + x - (nb + nx)) * nz + (z - nb);
    if (xin && z >= nb - H && z < nb) return 2 * H * nz + (x - nb) * H + (z - (nb - H));
    if (xin && z >= nb + nz && z < nb + nz + H) return 2 * H * nz + (nx + x - nb) * H + (z - (nb + nz));
    return -1;
}
inline int strip_cells(int nx, int nz, int H) { return 2 * H * (nx + nz); }

// One receiver of a tile, staged in shared memory by the step kernel's producer.
struct RecEntry {
    int z;          // extended row of its cell
    int ir;         // receiver index (trace row)
    float tr;       // trace sample of this step (backward), unused when recording
};

// One CTA's work item: everything the step kernel's producer needs to decode
// the tile's step and issue its TMA boxes, so that the issue waits on this one
// 80-byte load only (the descriptor and tables follow in parallel).
struct TileRef {
    int slot;            // index into the descriptor array
    int vd_x, vd_buf;    // where the tile's (v dt)^2 box is loaded from: column and
                         // field-pool buffer (the slot's own copy, or the model's
                         // table shared by every shot on that model)
    int has_pts;         // the tile holds receiver cells
    int x0, z0;          // first column and row of the tile
    int field_base;      // first field buffer of the shot's slot
    int nt;              // time samples of the shot's time axis
    long long g0;        // global step at which the job's forward step 0 runs
    int total_steps;     // steps of the job
    int si;              // store interval
    const float* wx;     // the shot's x taper (nxe)
    const float* wz;     // the model's z taper (ldz)
    int flags;           // ShotFlags of the job
    int nxe, nze;        // extended grid of the shot
    int has_src;         // the tile holds the source cell
};
static_assert(sizeof(TileRef) == 80, "TileRef layout");

// Host-side construction of a TileRef from the slot's descriptor.
inline TileRef make_tile_ref(const ShotDesc& d, int slot, int tx, int tz, int tile_x, bool has_pts,
                             int nbuf = kFieldBuffers, bool source_tile = false, int band_z0 = 0,
                             int band_x0 = 0) {
    TileRef r{};
    r.slot = slot;
    r.has_pts = has_pts ? 1 : 0;
    r.x0 = band_x0 + tx * tile_x;
    r.z0 = band_z0 + tz * kTileZ;
    r.field_base = d.field_slot * nbuf;
    r.vd_x = r.x0;
    r.vd_buf = r.field_base + 2;
    r.nt = d.nt;
    r.g0 = d.g0;
    r.total_steps = d.total_steps;
    r.si = d.si;
    r.wx = d.wx;
    r.wz = d.wz;
    r.flags = d.flags | (source_tile ? kFlagSourceTile : 0);
    r.nxe = d.nxe;
    r.nze = d.nze;
    r.has_src = d.src_x >= r.x0 && d.src_x < r.x0 + tile_x && d.src_z >= r.z0 && d.src_z < r.z0 + kTileZ;
    return r;
}

// The float value of a BF16 bit pattern (exact: BF16 is the top half of a float).
RTMB_HOST_DEVICE inline float bf16_bits_to_float(uint16_t b) {
    const uint32_t u = (uint32_t)b << 16;
#ifdef __CUDA_ARCH__
    return __uint_as_float(u);
#else
    float f;
    std::memcpy(&f, &u, sizeof f);
    return f;
#endif
}

// Error bits written by the kernels into the engine's device error word.
enum DeviceError : int {
    kErrTmaTimeout = 1,
    kErrBadTile = 2,
    kErrBarrierTimeout = 4,
};

}  // namespace rtmb
