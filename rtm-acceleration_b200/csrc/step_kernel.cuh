// step_kernel.cuh -- the fused leapfrog time step for sm_100a.
//
// A persistent, warp-specialised kernel advances every tile (128 rows x TX
// columns of one shot) of the tile list by one time step.  What the reference
// does in five passes per step (fd_time_step, inject_*, apply_sponge,
// save_snapshot / imaging; reference src/rtm/forward.cpp:29-125,
// backward.cpp:20-75, imaging.cpp:25-40) happens here in one:
//
//   1. a producer warp streams the CTA's tiles through a ring of shared-memory
//      stages: per tile it stages the shot descriptor and taper weights and one
//      lane issues 3D TMA box loads of p^n (tile + stencil halo), p^{n-1} and the
//      shot's (v dt)^2 against the stage's "full" mbarrier;
//   2. eight consumer warps wait on "full", each thread owns 4 consecutive depth
//      cells (a float4) of its share of the tile's columns and evaluates the
//      order-2H Laplacian
//      from shared memory, then releases the stage on its "empty" mbarrier;
//   3. p^{n+1} = w (2 p^n - w p^{n-1} + vdt2 lap) + injection, written in place
//      over p^{n-1} (only the owning thread touches that cell, so two time
//      levels suffice and there is no read/write race);
//   4. on stored steps the forward pass writes the interior snapshot (FP32, or
//      BF16/FP16 with a power-of-two scale per 128-cell column segment) and the
//      backward pass correlates with the stored snapshot (I += f b, S += f^2),
//      either straight into the running image or into per-shot compensated sums.
//
// Successive step launches are programmatic dependent launches: a step's CTAs
// wait in griddepcontrol.wait for the previous step to complete, so launch
// processing overlaps the previous step's tail.
//
// Arithmetic: with EXACT=true every float operation is an IEEE round-to-nearest
// add or multiply (no FMA contraction) in the same order as the reference's
// -O2 x86-64 build, so the result is bit-identical to the reference CPU engine.
// The damping identity used for the in-place update is the one the reference's
// cpu-opt engine relies on (reference src/cpu_opt/cpu_opt.cpp:125-170): the
// reference damps p^n in place after the step and reads it as p^{n-1} next step;
// here the stored value is read and damped on the fly, the same single multiply.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "internal.hpp"

namespace rtmb {

struct StepParams {
    void* fields;                 // field pool base (T*)
    long long slot_stride;        // elements per slot (two buffers)
    long long buf_stride;         // elements per buffer
    int ldz;                      // column pitch (elements)
    int ntiles;
    const ShotDesc* descs;
    const TileRef* tiles;
    const long long* step_counter;  // global step of the first launch of a chunk
    int step_offset;                // this launch's offset within the chunk
    int* error_word;
    int nstage;                     // pipeline stages (2..4) in dynamic shared memory
    int pdl;                        // host side: launch as a programmatic dependent launch
    int stall_tile;                 // failure-detection test: this tile is never produced (-1: none)
    int march_m;                    // march kernel: strip length in units of 2H+1 columns
    int nbuf;                       // field buffers per slot (kFieldBuffers or kReconBuffers)
    int spare;                      // ring kernel: leave one CTA slot per SM free, so that the
                                    // next step's CTAs become resident before this step ends
};

// ---------------------------------------------------------------- arithmetic
template <typename T, bool EXACT>
struct Arith {
    static __device__ __forceinline__ T add(T a, T b) { return a + b; }
    static __device__ __forceinline__ T sub(T a, T b) { return a - b; }
    static __device__ __forceinline__ T mul(T a, T b) { return a * b; }
};
template <>
struct Arith<float, true> {
    static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
    static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
    static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
};

// ------------------------------------------------------------ vector access
__device__ __forceinline__ void ld4(const float* p, float (&r)[4]) {
    const float4 t = *reinterpret_cast<const float4*>(p);
    r[0] = t.x; r[1] = t.y; r[2] = t.z; r[3] = t.w;
}
__device__ __forceinline__ void ld4(const double* p, double (&r)[4]) {
    const double2 a = reinterpret_cast<const double2*>(p)[0];
    const double2 b = reinterpret_cast<const double2*>(p)[1];
    r[0] = a.x; r[1] = a.y; r[2] = b.x; r[3] = b.y;
}
__device__ __forceinline__ void ldg4(const float* p, float (&r)[4]) {
    const float4 t = __ldg(reinterpret_cast<const float4*>(p));
    r[0] = t.x; r[1] = t.y; r[2] = t.z; r[3] = t.w;
}
__device__ __forceinline__ void st4(float* p, const float (&r)[4]) {
    *reinterpret_cast<float4*>(p) = make_float4(r[0], r[1], r[2], r[3]);
}
__device__ __forceinline__ void st4(double* p, const double (&r)[4]) {
    reinterpret_cast<double2*>(p)[0] = make_double2(r[0], r[1]);
    reinterpret_cast<double2*>(p)[1] = make_double2(r[2], r[3]);
}
// streaming (evict-first) variants for write-once / read-once snapshot data
__device__ __forceinline__ void st4cs(float* p, const float (&r)[4]) {
    __stcs(reinterpret_cast<float4*>(p), make_float4(r[0], r[1], r[2], r[3]));
}
__device__ __forceinline__ void st4cs(double* p, const double (&r)[4]) {
    __stcs(reinterpret_cast<double2*>(p), make_double2(r[0], r[1]));
    __stcs(reinterpret_cast<double2*>(p) + 1, make_double2(r[2], r[3]));
}
__device__ __forceinline__ void ld4cs(const float* p, float (&r)[4]) {
    const float4 t = __ldcs(reinterpret_cast<const float4*>(p));
    r[0] = t.x; r[1] = t.y; r[2] = t.z; r[3] = t.w;
}
__device__ __forceinline__ void ld4cs(const double* p, double (&r)[4]) {
    const double2 a = __ldcs(reinterpret_cast<const double2*>(p));
    const double2 b = __ldcs(reinterpret_cast<const double2*>(p) + 1);
    r[0] = a.x; r[1] = a.y; r[2] = b.x; r[3] = b.y;
}

// Explicit global-space accesses for the consumers' field, snapshot and image
// traffic: the stores are ordered only among themselves (no memory clobber), so
// the compiler may issue the next column's shared-memory loads ahead of them.
__device__ __forceinline__ size_t gaddr(const void* p) { return __cvta_generic_to_global(p); }
__device__ __forceinline__ void stg4(float* p, const float (&r)[4]) {
    asm volatile("st.global.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(gaddr(p)), "f"(r[0]), "f"(r[1]), "f"(r[2]),
                 "f"(r[3]));
}
__device__ __forceinline__ void stg4(double* p, const double (&r)[4]) {
    asm volatile("st.global.v2.f64 [%0], {%1, %2};" ::"l"(gaddr(p)), "d"(r[0]), "d"(r[1]));
    asm volatile("st.global.v2.f64 [%0], {%1, %2};" ::"l"(gaddr(p + 2)), "d"(r[2]), "d"(r[3]));
}
__device__ __forceinline__ void stg4cs(float* p, const float (&r)[4]) {
    asm volatile("st.global.cs.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(gaddr(p)), "f"(r[0]), "f"(r[1]), "f"(r[2]),
                 "f"(r[3]));
}
__device__ __forceinline__ void stg4cs(double* p, const double (&r)[4]) {
    asm volatile("st.global.cs.v2.f64 [%0], {%1, %2};" ::"l"(gaddr(p)), "d"(r[0]), "d"(r[1]));
    asm volatile("st.global.cs.v2.f64 [%0], {%1, %2};" ::"l"(gaddr(p + 2)), "d"(r[2]), "d"(r[3]));
}
__device__ __forceinline__ void stg_u2cs(void* p, uint2 v) {
    asm volatile("st.global.cs.v2.u32 [%0], {%1, %2};" ::"l"(gaddr(p)), "r"(v.x), "r"(v.y));
}
__device__ __forceinline__ void stg1(float* p, float v) {
    asm volatile("st.global.f32 [%0], %1;" ::"l"(gaddr(p)), "f"(v));
}
// Loads of data this launch does not write from another thread (image sums are
// read and written by their owning thread only).
__device__ __forceinline__ void ldg4(const float* p, float (&r)[4], int) {
    asm("ld.global.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(r[0]), "=f"(r[1]), "=f"(r[2]), "=f"(r[3]) : "l"(gaddr(p)));
}
__device__ __forceinline__ void ldg4(const double* p, double (&r)[4], int) {
    asm("ld.global.v2.f64 {%0, %1}, [%2];" : "=d"(r[0]), "=d"(r[1]) : "l"(gaddr(p)));
    asm("ld.global.v2.f64 {%0, %1}, [%2];" : "=d"(r[2]), "=d"(r[3]) : "l"(gaddr(p + 2)));
}

// 2^e as a float, exact for e in [-126, 127].
__device__ __forceinline__ float pow2f(int e) { return __int_as_float((e + 127) << 23); }

// Four BF16 words (8 bytes, the compensation words of a 4-row group) to and
// from T, rounding to nearest even on the way out.
template <typename T>
__device__ __forceinline__ void ldg_bf16x4(const uint16_t* p, T (&r)[4]) {
    uint32_t a, b;
    asm("ld.global.v2.u32 {%0, %1}, [%2];" : "=r"(a), "=r"(b) : "l"(gaddr(p)));
    r[0] = (T)__uint_as_float(a << 16);
    r[1] = (T)__uint_as_float(a & 0xffff0000u);
    r[2] = (T)__uint_as_float(b << 16);
    r[3] = (T)__uint_as_float(b & 0xffff0000u);
}
template <typename T>
__device__ __forceinline__ void stg_bf16x4(uint16_t* p, const T (&r)[4]) {
    const __nv_bfloat162 a = __floats2bfloat162_rn((float)r[0], (float)r[1]);
    const __nv_bfloat162 b = __floats2bfloat162_rn((float)r[2], (float)r[3]);
    asm volatile("st.global.v2.u32 [%0], {%1, %2};" ::"l"(gaddr(p)), "r"(*reinterpret_cast<const uint32_t*>(&a)),
                 "r"(*reinterpret_cast<const uint32_t*>(&b)));
}

// ------------------------------------------------------- TMA and mbarriers
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// The same test, but a thread whose phase is not complete is suspended (it
// issues nothing) until the phase completes or about `hint_ns` pass, so a
// waiting warp leaves the issue slots to the warps that have work.
__device__ __forceinline__ bool mbar_try_wait_sleep(uint64_t* bar, uint32_t parity, uint32_t hint_ns) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity), "r"(hint_ns)
        : "memory");
    return ok != 0;
}
constexpr uint32_t kSleepHintNs = 20000;
// Plain (non-multicast) tiled TMA load of a 3D box from this GPU's own memory.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1,
                                            int c2) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_addr(bar)), "r"(c0), "r"(c1), "r"(c2)
        : "memory");
}

// Wall-clock bound of every wait in the step kernel (globaltimer, ns).  A wait
// that runs out sets an error bit and returns, so the kernel ends and the host
// reports RTM_B200_ETIMEOUT instead of the GPU hanging.
constexpr unsigned long long kWaitNs = 1000000000ull;   // 1 s

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait: gives up after `ns` nanoseconds and reports it in the error word.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int* err, unsigned long long ns) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (!mbar_try_wait(bar, parity)) {
        if (global_ns() - t0 > ns) {
            atomicOr(err, kErrTmaTimeout);
            return false;
        }
    }
    return true;
}

// Halo depth in rows, rounded up to 4 so the TMA box starts 16-byte aligned.
template <int H>
struct Halo {
    static constexpr int HP = (H + 3) & ~3;
};

// One shared-memory stage of the pipelined step kernel:
//   [0, 128)      TileInfo: what the tile does this step (written by the producer)
//   [128, ...)    the tile's ShotDesc
//   [WX_OFF, ..)  taper weights wx of the tile's TX columns
//   [WZ_OFF, ..)  taper weights wz of the tile's 128 rows
//   [CS_OFF, ..)  receiver-cell offsets col_start[x0 .. x0+TX] (unstaged receivers)
//   [RCS_OFF, ..) staged receivers: per-column offsets into the entries below
//   [REC_OFF, ..) staged receivers: RecEntry {row, index, trace sample}
//   [PC_OFF, ..)  TMA box of p^n with the stencil halo      (SZ x SX)
//   [PP_OFF, ..)  TMA box of p^{n-1}                         (128 x TX)
//   [VD_OFF, ..)  TMA box of the shot's (v dt)^2             (128 x TX)
struct alignas(16) TileInfo {
    int active, fwd, first, it, cur, x0, z0, tz;
    int do_snap, do_image, ksnap, has_pts, rec_staged;
    int glog;   // log2 of the lanes per column of the band (step kernel)
    int plain;  // step kernel: no cell of the tile is masked, injects or records
    int unitw;  // step kernel: every live cell of the tile has sponge weight exactly 1
    int prv;    // slot buffer holding p^{n-1} (written with p^{n+1}); cur holds p^n
    int src;    // reconstruction, stored backward steps: slot buffer holding the
                // source field at the imaged level (-1: images read snapshots)
    int recon;  // a tile of the source field running backwards
    int strip;  // forward pass with reconstruction: store the boundary strip
};
static_assert(sizeof(TileInfo) <= 128, "TileInfo fits its block of the stage header");

__host__ __device__ constexpr int ilog2(int v) { return v <= 1 ? 0 : 1 + ilog2(v / 2); }

constexpr int kTileRec = 128;   // receivers a tile can stage in shared memory

// NCW consumer warps share a tile of 128 rows x TX_ columns.
template <typename T, int H, int NCW, int TX_>
struct TileShape {
    static constexpr int HP = Halo<H>::HP;
    static constexpr int TX = TX_;
    static constexpr int SZ = kTileZ + 2 * HP;   // rows of the p^n box
    static constexpr int SX = TX + 2 * H;        // columns of the p^n box
    static constexpr int PC_BYTES = SZ * SX * (int)sizeof(T);
    static constexpr int BOX_BYTES = kTileZ * TX * (int)sizeof(T);
    static constexpr int INFO_OFF = 0;
    static constexpr int DESC_OFF = 128;
    static constexpr int WX_OFF = 512;
    static constexpr int WZ_OFF = WX_OFF + 128;
    static constexpr int CS_OFF = WZ_OFF + kTileZ * 4;
    static constexpr int RCS_OFF = 1408;
    static constexpr int REC_OFF = RCS_OFF + 256;
    static constexpr int HDR = REC_OFF + kTileRec * (int)sizeof(RecEntry);
    static constexpr int PC_OFF = HDR;
    static constexpr int PP_OFF = PC_OFF + ((PC_BYTES + 127) & ~127);
    static constexpr int VD_OFF = PP_OFF + ((BOX_BYTES + 127) & ~127);
    static constexpr int STAGE = VD_OFF + ((BOX_BYTES + 127) & ~127);
    static_assert(TX <= 32, "wx staging holds at most 32 columns");
    static_assert(CS_OFF + 4 * (TX + 1) <= RCS_OFF, "stage header overflow");
    static_assert(4 * (TX + 1) <= REC_OFF - RCS_OFF, "staged receiver offsets overflow");
    static_assert(HDR % 128 == 0, "TMA boxes must start 128-byte aligned");
    static_assert(INFO_OFF + sizeof(TileInfo) <= DESC_OFF, "tile info overflows its block");
    static_assert(DESC_OFF + sizeof(ShotDesc) <= WX_OFF, "descriptor overflows its block");
    static_assert(STAGE % 128 == 0 && DESC_OFF % 16 == 0, "stages and the descriptor copy are 16-byte aligned");
};

// Decodes a snapshot value group (4 rows).
template <typename T>
__device__ __forceinline__ void load_snapshot4(const ShotDesc& d, size_t cell, size_t eidx, T (&f)[4]) {
    if (d.snap_type == kSnapF32 || d.snap_type == kSnapF64) {
        ld4cs(reinterpret_cast<const T*>(d.snap) + cell, f);
    } else {
        const uint2 packed =
            __ldcs(reinterpret_cast<const uint2*>(reinterpret_cast<const uint16_t*>(d.snap) + cell));
        const float sc = pow2f((int)__ldg(d.snap_exp + eidx));
        float2 a, b;
        if (d.snap_type == kSnapF16) {
            a = __half22float2(*reinterpret_cast<const __half2*>(&packed.x));
            b = __half22float2(*reinterpret_cast<const __half2*>(&packed.y));
        } else {
            a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&packed.x));
            b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&packed.y));
        }
        f[0] = (T)(a.x * sc); f[1] = (T)(a.y * sc); f[2] = (T)(b.x * sc); f[3] = (T)(b.y * sc);
    }
}

// ------------------------------------------------------ column arithmetic
// One column of 4 rows: Laplacian from the p^n box, leapfrog with the sponge,
// before injection and masking.  Generic scalar form (used for double).
template <typename T, int H, bool EXACT, int SZ, int HP>
struct ColumnMath {
    static __device__ __forceinline__ void run(const T* col, const T (&pp)[4], const T (&vd)[4], float wxv,
                                               const float (&wz)[4], T c0, const float* cxs, const float* czs,
                                               bool first, T (&val)[4]) {
        using A = Arith<T, EXACT>;
        // coefficients 0..H from the descriptor's 16-byte aligned rows, as float4s
        constexpr int kChunks = (H + 4) / 4;
        float cx[4 * kChunks], cz[4 * kChunks];
#pragma unroll
        for (int c = 0; c < kChunks; ++c) {
            const float4 a = reinterpret_cast<const float4*>(cxs)[c];
            const float4 b = reinterpret_cast<const float4*>(czs)[c];
            cx[4 * c] = a.x; cx[4 * c + 1] = a.y; cx[4 * c + 2] = a.z; cx[4 * c + 3] = a.w;
            cz[4 * c] = b.x; cz[4 * c + 1] = b.y; cz[4 * c + 2] = b.z; cz[4 * c + 3] = b.w;
        }
        // First step of a pass: p^n = p^{n-1} = 0 and the update below gives +0
        // in every rounding step (2*0 - 0*w = +0, +0 + vd*(+-0) = +0, +0*w = +0),
        // so the boxes (not loaded for this step) are not read.
        if (first) {
#pragma unroll
            for (int q = 0; q < 4; ++q) val[q] = (T)0;
            return;
        }
        T zz[4 + 2 * HP];
#pragma unroll
        for (int g = 0; g < (4 + 2 * HP) / 4; ++g) {
            T tt[4];
            ld4(col - HP + 4 * g, tt);
#pragma unroll
            for (int q = 0; q < 4; ++q) zz[4 * g + q] = tt[q];
        }
        // FP32 with FMA: the explicit fused form of the packed pair path
        // (column_pair_f32), so every FP32 ring variant computes the same bits.
        constexpr bool kFused = !EXACT && sizeof(T) == 4;
        T lap[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) lap[q] = A::mul(c0, zz[HP + q]);
#pragma unroll
        for (int k = 1; k <= H; ++k) {
            T xm[4], xp[4];
            ld4(col - k * SZ, xm);
            ld4(col + k * SZ, xp);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const T ax = A::add(xp[q], xm[q]);
                const T az = A::add(zz[HP + q + k], zz[HP + q - k]);
                if constexpr (kFused)
                    lap[q] = __fmaf_rn((float)cz[k], az, __fmaf_rn((float)cx[k], ax, lap[q]));
                else
                    lap[q] = A::add(lap[q], A::add(A::mul((T)cx[k], ax), A::mul((T)cz[k], az)));
            }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const T w = (T)__fmul_rn(wxv, wz[q]);
            const T prev = A::mul(pp[q], w);
            if constexpr (kFused) {
                val[q] = __fmul_rn(__fmaf_rn(vd[q], lap[q], __fmaf_rn(2.0f, zz[HP + q], -prev)), w);
            } else {
                const T s = A::add(A::sub(A::mul((T)2, zz[HP + q]), prev), A::mul(vd[q], lap[q]));
                val[q] = A::mul(s, w);
            }
        }
    }
};


// ------------------------------------------------------- column epilogue
// Everything after the stencil arithmetic for one column of 4 rows per lane:
// the zero outer ring, source and receiver injection (or trace recording), the
// store of p^{n+1}, and on stored steps the snapshot store (forward) or the
// imaging update (backward).  Shared by both step kernels.  Receivers: with
// t.rec_staged, re[rkb..rke) are the column's staged receivers; otherwise
// d.pts[rkb..rke) are its receiver cells in global memory.
template <typename T, int H, bool EXACT>
__device__ __forceinline__ void column_epilogue(const ShotDesc& d, const TileInfo& t, int x, int zr, int lane,
                                                bool lane_in, bool lane_snap, T (&val)[4], const T (&vd)[4],
                                                const T (&fs)[4], T (&Iv)[4], T (&Sv)[4], int rkb, int rke,
                                                const RecEntry* __restrict__ re, T* __restrict__ pcur,
                                                T* __restrict__ pnext, int ldz, int G) {
    using A = Arith<T, EXACT>;
    const bool first = t.first;
    const bool do_snap = t.do_snap, do_image = t.do_image;
    // Plain tile on an unstored step (the common case): every cell of the tile is
    // live and interior to the zero ring, so the store is all there is.
    if (t.plain && !do_snap && !do_image) {
        stg4(pnext + (uint32_t)x * (uint32_t)ldz + zr, val);
        if (first) {
            const T z4[4] = {0, 0, 0, 0};
            stg4(pcur + (uint32_t)x * (uint32_t)ldz + zr, z4);
        }
        return;
    }
    const int nxe = d.nxe, nze = d.nze, nb = d.nb, nx = d.nx, lds = d.lds, zs0 = d.zs0;
    const int it = t.it;
    const bool fwd = t.fwd;
    const int snap_type = d.snap_type;
    const bool col_live = x < nxe;
    const bool col_int = (x >= nb) && (x < nb + nx);
    const uint32_t ic = (uint32_t)(x - nb) * (uint32_t)lds + (uint32_t)(zr - zs0);
    if (!t.plain) {
        // the outer H-ring of the grid (and rows/columns past it) stays 0
        const bool col_ok = (x >= H) && (x < nxe - H);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const bool row_ok = (zr + q >= H) && (zr + q < nze - H);
            val[q] = (col_ok && row_ok) ? val[q] : (T)0;
        }

        // Injection at cells whose taper is exactly 1, so adding after the
        // damping matches the reference's inject-then-damp order bit for bit.
        if (fwd && x == d.src_x) {
            const T amp = (T)__ldg(d.wavelet + it);
#pragma unroll
            for (int q = 0; q < 4; ++q)
                if (zr + q == d.src_z) val[q] = A::add(val[q], A::mul(vd[q], amp));
        }
        // Receiver cells of this column: inject (backward) or record (forward
        // modelling).  Several receivers on one cell add in ascending ir order,
        // like the reference's sequential loop (backward.cpp:20-27).
        if (t.has_pts) {
            if (t.rec_staged) {
                for (int k = rkb; k < rke; ++k) {
                    const RecEntry e = re[k];
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        if (e.z != zr + q) continue;
                        if (fwd)
                            stg1(d.rec_out + (size_t)e.ir * d.nt + it, (float)val[q]);
                        else
                            val[q] = A::add(val[q], A::mul(vd[q], (T)e.tr));
                    }
                }
            } else {
                for (int j = rkb; j < rke; ++j) {
                    const PointEntry e = d.pts[j];
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        if (e.z != zr + q) continue;
                        for (int r = 0; r < e.ir_count; ++r) {
                            const int ir = __ldg(d.pts_ir + e.ir_begin + r);
                            if (fwd) {
                                stg1(d.rec_out + (size_t)ir * d.nt + it, (float)val[q]);
                            } else {
                                const T tr = (T)__ldg(d.traces + (size_t)ir * d.trace_nt + it);
                                val[q] = A::add(val[q], A::mul(vd[q], tr));
                            }
                        }
                    }
                }
            }
        }
    }

    if (!t.plain && (t.recon || t.strip)) {
        // Source reconstruction.  A tile of the source field running backwards
        // keeps its update on the interior, takes the band of H cells around it
        // from the strip the forward pass stored for this level, and clears
        // every other cell (nothing reads them).  A forward tile stores its
        // band cells of level it+1 into that level's strip.
        const int H_ = H;
        const size_t lev = (size_t)(t.recon ? t.it - 2 : t.it) * (size_t)d.bsize;   // level - 1
        float* strip = reinterpret_cast<float*>(d.snap) + lev;
        const bool xin = x >= nb && x < nb + nx;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int z = zr + q;
            const int bi = strip_index(x, z, nb, nx, d.nz, H_);
            if (t.recon) {
                if (!(xin && z >= nb && z < nb + d.nz)) val[q] = bi >= 0 ? (T)__ldg(strip + bi) : (T)0;
            } else if (bi >= 0 && lane_in && col_live) {
                stg1(strip + bi, (float)val[q]);
            }
        }
    }

    if (lane_in && col_live) {
        stg4(pnext + (uint32_t)x * (uint32_t)ldz + zr, val);
        if (first) {   // p^n of the first step is zero: clear the other level too
            const T z4[4] = {0, 0, 0, 0};
            stg4(pcur + (uint32_t)x * (uint32_t)ldz + zr, z4);
        }
    }

    // Power-of-two scale of a reduced-precision snapshot, one per (snapshot,
    // column, 128-row segment): the maximum over the G lanes of the column,
    // taken by every lane of the warp (the shuffles need all 32).
    float amax_col = 0.f;
    if (do_snap && (snap_type == kSnapBF16 || snap_type == kSnapF16)) {
        float a = 0.f;
        if (col_int && lane_snap)
#pragma unroll
            for (int q = 0; q < 4; ++q) a = fmaxf(a, fabsf((float)val[q]));
        if (G == 32) {
            // one warp-wide reduction: for non-negative floats the order of
            // the bit patterns as unsigned integers is the order of the values
            a = __uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(a)));
        } else {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
                if (o < G) a = fmaxf(a, __shfl_xor_sync(0xffffffffu, a, o));
        }
        amax_col = a;
    }

    if (col_int && (do_snap || do_image)) {
        if (do_snap) {
            const size_t cell = (size_t)t.ksnap * nx * lds + ic;
            if (snap_type == kSnapF32 || snap_type == kSnapF64) {
                if (lane_snap) stg4cs(reinterpret_cast<T*>(d.snap) + cell, val);
            } else {
                const float amax = amax_col;
                int e = 0;
                if (amax > 0.f) {
                    // amax <= 2^e from the exponent field (subnormals: e = -126)
                    const int ex = (__float_as_int(amax) >> 23) & 0xff;
                    e = ex == 0 ? -126 : ex - 126;
                    e -= 15;                   // scaled max <= 2^15
                    e = e < -126 ? -126 : (e > 127 ? 127 : e);
                }
                const size_t eidx = ((size_t)t.ksnap * nx + (x - nb)) * d.ntz + t.tz;
                if ((lane & (G - 1)) == 0) d.snap_exp[eidx] = (int8_t)e;
                if (lane_snap) {
                    const float inv = pow2f(-e);
                    uint2 packed;
                    if (snap_type == kSnapF16) {
                        const __half2 a = __floats2half2_rn((float)val[0] * inv, (float)val[1] * inv);
                        const __half2 b = __floats2half2_rn((float)val[2] * inv, (float)val[3] * inv);
                        packed.x = *reinterpret_cast<const uint32_t*>(&a);
                        packed.y = *reinterpret_cast<const uint32_t*>(&b);
                    } else {
                        const __nv_bfloat162 a = __floats2bfloat162_rn((float)val[0] * inv, (float)val[1] * inv);
                        const __nv_bfloat162 b = __floats2bfloat162_rn((float)val[2] * inv, (float)val[3] * inv);
                        packed.x = *reinterpret_cast<const uint32_t*>(&a);
                        packed.y = *reinterpret_cast<const uint32_t*>(&b);
                    }
                    stg_u2cs(reinterpret_cast<uint16_t*>(d.snap) + cell, packed);
                }
            }
        }
        if (do_image && lane_snap) {
            T* img = reinterpret_cast<T*>(d.img) + ic;
            T* ill = reinterpret_cast<T*>(d.ill) + ic;
            if (d.acc_mode == kAccPlain) {
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    Iv[q] = A::add(Iv[q], A::mul(fs[q], val[q]));
                    Sv[q] = A::add(Sv[q], A::mul(fs[q], fs[q]));
                }
            } else {
                // Kahan: sum + (term - comp), comp tracks the lost low part.
                // The compensation words are kept in BF16 (FP32 engines only):
                // |comp| stays below about one ulp of the sum, so storing it
                // with an 8-bit mantissa costs at most 2^-10 ulp(sum) per
                // update, about 0.04 ulp after 2000 stored steps, and saves a
                // quarter of a stored backward step's imaging traffic.
                uint16_t* imc = reinterpret_cast<uint16_t*>(d.img_c) + ic;
                uint16_t* ilc = reinterpret_cast<uint16_t*>(d.ill_c) + ic;
                T Ic[4], Sc[4];
                ldg_bf16x4(imc, Ic);
                ldg_bf16x4(ilc, Sc);
                using E = Arith<T, true>;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const T yi = E::sub(E::mul(fs[q], val[q]), Ic[q]);
                    const T ti = E::add(Iv[q], yi);
                    Ic[q] = E::sub(E::sub(ti, Iv[q]), yi);
                    Iv[q] = ti;
                    const T ys = E::sub(E::mul(fs[q], fs[q]), Sc[q]);
                    const T ts = E::add(Sv[q], ys);
                    Sc[q] = E::sub(E::sub(ts, Sv[q]), ys);
                    Sv[q] = ts;
                }
                stg_bf16x4(imc, Ic);
                stg_bf16x4(ilc, Sc);
            }
            stg4(img, Iv);
            stg4(ill, Sv);
        }
    }
}

// ------------------------------------------------- paired FP32 arithmetic
// Two FP32 values per operation.  PK<true> issues one packed sm_100
// instruction (add/mul/fma .f32x2) per operation; PK<false> issues two scalar
// __fadd_rn / __fmul_rn / __fmaf_rn.  The IEEE (bit-identical) path uses the
// scalar form: every operation of the reference is then a separately rounded
// add or multiply that the optimiser never contracts.  The FMA path uses the
// packed form.  add and mul are written as PTX with an explicit .rn modifier,
// which the optimiser does not fuse either.
template <bool PACK>
struct PK;
template <>
struct PK<true> {
    static __device__ __forceinline__ float2 add(float2 a, float2 b) {
        float2 d;
        asm("{\n\t.reg .b64 ra, rb, rd;\n\t"
            "mov.b64 ra, {%2, %3};\n\t"
            "mov.b64 rb, {%4, %5};\n\t"
            "add.rn.f32x2 rd, ra, rb;\n\t"
            "mov.b64 {%0, %1}, rd;\n\t}"
            : "=f"(d.x), "=f"(d.y)
            : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
        return d;
    }
    static __device__ __forceinline__ float2 mul(float2 a, float2 b) {
        float2 d;
        asm("{\n\t.reg .b64 ra, rb, rd;\n\t"
            "mov.b64 ra, {%2, %3};\n\t"
            "mov.b64 rb, {%4, %5};\n\t"
            "mul.rn.f32x2 rd, ra, rb;\n\t"
            "mov.b64 {%0, %1}, rd;\n\t}"
            : "=f"(d.x), "=f"(d.y)
            : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
        return d;
    }
    static __device__ __forceinline__ float2 fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
};
template <>
struct PK<false> {
    static __device__ __forceinline__ float2 add(float2 a, float2 b) {
        return make_float2(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y));
    }
    static __device__ __forceinline__ float2 mul(float2 a, float2 b) {
        return make_float2(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y));
    }
    static __device__ __forceinline__ float2 fma(float2 a, float2 b, float2 c) {
        return make_float2(__fmaf_rn(a.x, b.x, c.x), __fmaf_rn(a.y, b.y, c.y));
    }
};
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 dup2(float a) { return make_float2(a, a); }

// One pair of adjacent columns (a, b = a + 1) of 4 rows per lane, FP32: the
// Laplacian and the leapfrog update with the sponge, before injection and
// masking.  The two columns share their x-neighbour loads: the box columns
// a-H .. b+H are each read once (2H loads for the pair instead of 4H), and the
// rows are processed two at a time (q = 0,1 and 2,3).
//
// EXACT: every operation is a separately rounded IEEE add or multiply in the
// reference's order (lap = c0 p; lap += cx (xp + xm) + cz (zp + zm) for k = 1..H;
// p' = w ((2p - w pp) + vd lap)).  Otherwise the same scheme with fused
// multiply-adds (lap = fma(cz, zp + zm, fma(cx, xp + xm, lap)); p' = w fma(vd,
// lap, fma(2, p, -w pp))), two rows per packed instruction.  unitw: every cell of the tile has
// sponge weight exactly 1, so the weight multiplies are the identity and are
// skipped (bit-identical).
template <int H, bool EXACT, int SZ, int HP>
__device__ __forceinline__ void column_pair_f32(const float* ca, const float* ppa_s, const float* vda_s, float wxa,
                                                float wxb, const float (&wz)[4], float c0, const float* cxs,
                                                const float* czs, bool unitw, float (&va)[4], float (&vb)[4]) {
    using P = PK<!EXACT>;
    constexpr int NZ = 4 + 2 * HP;   // rows of a column window: HP above, 4 own, HP below
    const float* cb = ca + SZ;
    float za[NZ], zb[NZ];
#pragma unroll
    for (int g = 0; g < NZ / 4; ++g) {
        ld4(ca - HP + 4 * g, *reinterpret_cast<float(*)[4]>(za + 4 * g));
        ld4(cb - HP + 4 * g, *reinterpret_cast<float(*)[4]>(zb + 4 * g));
    }
    float2 la[2], lb[2];
    const float2 c0p = dup2(c0);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        la[h] = P::mul(c0p, make_float2(za[HP + 2 * h], za[HP + 2 * h + 1]));
        lb[h] = P::mul(c0p, make_float2(zb[HP + 2 * h], zb[HP + 2 * h + 1]));
    }
    // x queue: L = column a-(k-1), R = column b+(k-1); they start at the centres
    float L[4], R[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) { L[q] = za[HP + q]; R[q] = zb[HP + q]; }
#pragma unroll
    for (int k = 1; k <= H; ++k) {
        float Lk[4], Rk[4];
        ld4(ca - k * SZ, Lk);
        ld4(cb + k * SZ, Rk);
        const float2 cxp = dup2(cxs[k]), czp = dup2(czs[k]);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int r = HP + 2 * h;   // first of the two rows of this pair
            // column a: x-k = Lk, x+k = R;  column b: x-k = L, x+k = Rk
            const float2 axa = P::add(make_float2(R[2 * h], R[2 * h + 1]), make_float2(Lk[2 * h], Lk[2 * h + 1]));
            const float2 axb = P::add(make_float2(Rk[2 * h], Rk[2 * h + 1]), make_float2(L[2 * h], L[2 * h + 1]));
            float2 aza, azb;
            if ((k & 1) == 0) {   // rows r+-k, r+1+-k are aligned register pairs
                aza = P::add(make_float2(za[r + k], za[r + 1 + k]), make_float2(za[r - k], za[r + 1 - k]));
                azb = P::add(make_float2(zb[r + k], zb[r + 1 + k]), make_float2(zb[r - k], zb[r + 1 - k]));
            } else {              // odd shift: form the sums from single rows
                aza = make_float2(__fadd_rn(za[r + k], za[r - k]), __fadd_rn(za[r + 1 + k], za[r + 1 - k]));
                azb = make_float2(__fadd_rn(zb[r + k], zb[r - k]), __fadd_rn(zb[r + 1 + k], zb[r + 1 - k]));
            }
            if (EXACT) {
                la[h] = P::add(la[h], P::add(P::mul(cxp, axa), P::mul(czp, aza)));
                lb[h] = P::add(lb[h], P::add(P::mul(cxp, axb), P::mul(czp, azb)));
            } else {
                la[h] = P::fma(czp, aza, P::fma(cxp, axa, la[h]));
                lb[h] = P::fma(czp, azb, P::fma(cxp, axb, lb[h]));
            }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) { L[q] = Lk[q]; R[q] = Rk[q]; }
    }
    // p' = w ((2p - w pp) + vd lap); p^{n-1} and (v dt)^2 of the pair are read
    // only now (column b follows column a at kTileZ floats in both boxes)
    float ppa[4], ppb[4], vda[4], vdb[4];
    ld4(ppa_s, ppa);
    ld4(ppa_s + kTileZ, ppb);
    ld4(vda_s, vda);
    ld4(vda_s + kTileZ, vdb);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const float2 wzp = make_float2(wz[2 * h], wz[2 * h + 1]);
        const float2 pa = make_float2(za[HP + 2 * h], za[HP + 2 * h + 1]);
        const float2 pb = make_float2(zb[HP + 2 * h], zb[HP + 2 * h + 1]);
        const float2 ppa2 = make_float2(ppa[2 * h], ppa[2 * h + 1]);
        const float2 ppb2 = make_float2(ppb[2 * h], ppb[2 * h + 1]);
        const float2 vda2 = make_float2(vda[2 * h], vda[2 * h + 1]);
        const float2 vdb2 = make_float2(vdb[2 * h], vdb[2 * h + 1]);
        float2 ra, rb;
        if (unitw) {
            if (EXACT) {
                ra = P::add(P::add(P::add(pa, pa), neg2(ppa2)), P::mul(vda2, la[h]));
                rb = P::add(P::add(P::add(pb, pb), neg2(ppb2)), P::mul(vdb2, lb[h]));
            } else {
                ra = P::fma(vda2, la[h], P::fma(dup2(2.0f), pa, neg2(ppa2)));
                rb = P::fma(vdb2, lb[h], P::fma(dup2(2.0f), pb, neg2(ppb2)));
            }
        } else {
            const float2 wa = P::mul(dup2(wxa), wzp), wb = P::mul(dup2(wxb), wzp);
            if (EXACT) {
                ra = P::mul(P::add(P::add(P::add(pa, pa), neg2(P::mul(ppa2, wa))), P::mul(vda2, la[h])), wa);
                rb = P::mul(P::add(P::add(P::add(pb, pb), neg2(P::mul(ppb2, wb))), P::mul(vdb2, lb[h])), wb);
            } else {
                ra = P::mul(P::fma(vda2, la[h], P::fma(dup2(2.0f), pa, neg2(P::mul(ppa2, wa)))), wa);
                rb = P::mul(P::fma(vdb2, lb[h], P::fma(dup2(2.0f), pb, neg2(P::mul(ppb2, wb)))), wb);
            }
        }
        va[2 * h] = ra.x; va[2 * h + 1] = ra.y;
        vb[2 * h] = rb.x; vb[2 * h + 1] = rb.y;
    }
}

// Which of a tile's work items (column pairs, or passes of packed columns) the
// consumer warp `warp` takes first: items go round-robin over the NCW warps
// from a first warp that moves with the tile's position, so that the warps that
// get one item more than the others change from tile to tile.
template <int NCW>
__device__ __forceinline__ int first_item(const TileInfo& t, int tx, int warp) {
    const int j = (int)(((unsigned)t.x0 / (unsigned)tx + (unsigned)t.tz) % NCW);
    const int f = warp - j;
    return f < 0 ? f + NCW : f;
}

// Full bands (32 lanes per column, the common case) of an FP32 tile: the tile's
// TX/2 pairs of adjacent columns go round-robin to the consumer warps; the two
// columns of a pair share their x-neighbour loads (column_pair_f32); the
// epilogue is the shared per-column one.
template <int H, bool EXACT, int NCW, int TX>
__device__ __forceinline__ void compute_tile_full_f32(const unsigned char* __restrict__ st, const TileInfo& t,
                                                      float* __restrict__ pcur, float* __restrict__ pnext,
                                                      const float* __restrict__ psrc, int ldz) {
    using S = TileShape<float, H, NCW, TX>;
    constexpr int HP = S::HP;
    const ShotDesc& d = *reinterpret_cast<const ShotDesc*>(st + S::DESC_OFF);
    const float* __restrict__ sm_pc = reinterpret_cast<const float*>(st + S::PC_OFF);
    const float* __restrict__ sm_pp = reinterpret_cast<const float*>(st + S::PP_OFF);
    const float* __restrict__ sm_vd = reinterpret_cast<const float*>(st + S::VD_OFF);
    const float* __restrict__ sm_wx = reinterpret_cast<const float*>(st + S::WX_OFF);
    const float* __restrict__ sm_wz = reinterpret_cast<const float*>(st + S::WZ_OFF);
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int nb = d.nb, nx = d.nx, lds = d.lds, zs0 = d.zs0;
    const int zr = t.z0 + 4 * lane;
    const bool lane_in = zr < d.nze;
    const bool lane_snap = lane_in && zr >= zs0 && zr < zs0 + lds;
    const bool first = t.first;
    const bool do_image = t.do_image;
    const bool unitw = t.unitw;
    float wz[4];
    {
        const float4 w4 = *reinterpret_cast<const float4*>(sm_wz + 4 * lane);
        wz[0] = w4.x; wz[1] = w4.y; wz[2] = w4.z; wz[3] = w4.w;
    }
    // Pairs of this warp: f, f + NCW, ... (a compile-time count when the
    // tile's pairs divide evenly over the warps).
    constexpr int kPairs = TX / 2;
    constexpr int kEven = kPairs % NCW == 0 ? kPairs / NCW : 0;
    const int f = first_item<NCW>(t, TX, warp);
    const int npr = kEven ? kEven : (kPairs - f + NCW - 1) / NCW;

    // Plain tile on an unstored step (most of the work): every cell is live,
    // inside the zero ring and free of injection and recording, so each pair
    // is computed and stored with nothing else.
    if (t.plain && !t.do_snap && !do_image) {
#pragma unroll
        for (int i = 0; i < (kEven ? kEven : 1); ++i) {
            for (int j = 0; j < (kEven ? 1 : npr); ++j) {
                const int la = 2 * (f + (i + j) * NCW);
                float va[4], vb[4];
                float* dst = pnext + (uint32_t)(t.x0 + la) * (uint32_t)ldz + zr;
                if (first) {
                    const float z4[4] = {0.f, 0.f, 0.f, 0.f};
                    float* cur = pcur + (uint32_t)(t.x0 + la) * (uint32_t)ldz + zr;
                    stg4(dst, z4);
                    stg4(dst + ldz, z4);
                    stg4(cur, z4);
                    stg4(cur + ldz, z4);
                } else {
                    column_pair_f32<H, EXACT, S::SZ, HP>(sm_pc + (la + H) * S::SZ + 4 * lane + HP,
                                                          sm_pp + la * kTileZ + 4 * lane,
                                                          sm_vd + la * kTileZ + 4 * lane, sm_wx[la], sm_wx[la + 1],
                                                          wz, d.c0, d.cx, d.cz, unitw, va, vb);
                    stg4(dst, va);
                    stg4(dst + ldz, vb);
                }
            }
        }
        return;
    }

    for (int j = 0; j < npr; ++j) {
        const int la = 2 * (f + j * NCW);
        float va[4], vb[4];
        if (first) {
            // p^n = p^{n-1} = 0 on the first step of a pass: the update is +0
            // in every rounding step, and the boxes were not loaded.
#pragma unroll
            for (int q = 0; q < 4; ++q) { va[q] = 0.f; vb[q] = 0.f; }
        } else {
            column_pair_f32<H, EXACT, S::SZ, HP>(sm_pc + (la + H) * S::SZ + 4 * lane + HP,
                                                  sm_pp + la * kTileZ + 4 * lane, sm_vd + la * kTileZ + 4 * lane,
                                                  sm_wx[la], sm_wx[la + 1], wz, d.c0, d.cx, d.cz, unitw, va, vb);
        }
        const RecEntry* re = reinterpret_cast<const RecEntry*>(st + S::REC_OFF);
        const int* off = t.has_pts
                             ? reinterpret_cast<const int*>(st + (t.rec_staged ? S::RCS_OFF : S::CS_OFF))
                             : nullptr;
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            const int lx = la + c, x = t.x0 + lx;
            float vd[4], fs[4], Iv[4], Sv[4];
            ld4(sm_vd + lx * kTileZ + 4 * lane, vd);   // injection weights (the epilogue's only use)
            if (do_image && lane_snap && x >= nb && x < nb + nx) {
                const uint32_t ic = (uint32_t)(x - nb) * (uint32_t)lds + (uint32_t)(zr - zs0);
                const size_t cell = (size_t)t.ksnap * nx * lds + ic;
                const size_t eidx = ((size_t)t.ksnap * nx + (x - nb)) * d.ntz + t.tz;
                if (psrc)   // reconstruction: the source field at the imaged level
                    ldg4(psrc + (uint32_t)x * (uint32_t)ldz + zr, fs, 0);
                else
                    load_snapshot4<float>(d, cell, eidx, fs);
                ldg4(reinterpret_cast<const float*>(d.img) + ic, Iv, 0);
                ldg4(reinterpret_cast<const float*>(d.ill) + ic, Sv, 0);
            }
            column_epilogue<float, H, EXACT>(d, t, x, zr, lane, lane_in, lane_snap, c ? vb : va, vd, fs, Iv, Sv,
                                             off ? off[lx] : 0, off ? off[lx + 1] : 0, re, pcur, pnext, ldz, 32);
        }
    }
}

// ------------------------------------------------------------- the tile
// Computes one tile after its boxes have landed in the stage.
template <typename T, int H, bool EXACT, int NCW, int TX>
__device__ __forceinline__ void compute_tile(const unsigned char* __restrict__ st, const TileInfo& t,
                                             T* __restrict__ pcur, T* __restrict__ pnext, const T* __restrict__ psrc,
                                             int ldz) {
    // FP32 full bands take the column-pair path, except in the 8-warp x
    // 16-column shape: it runs 2 CTAs of 9 warps per SM at 96 registers per
    // thread, where the per-column path below fits without spilling.
    if constexpr (sizeof(T) == 4 && !(NCW == 8 && TX == 16)) {
        if (t.glog == 5) {   // full band: the column-pair path
            compute_tile_full_f32<H, EXACT, NCW, TX>(st, t, pcur, pnext, psrc, ldz);
            return;
        }
    }
    using S = TileShape<T, H, NCW, TX>;
    constexpr int HP = S::HP;
    const ShotDesc& d = *reinterpret_cast<const ShotDesc*>(st + S::DESC_OFF);
    const T* __restrict__ sm_pc = reinterpret_cast<const T*>(st + S::PC_OFF);
    const T* __restrict__ sm_pp = reinterpret_cast<const T*>(st + S::PP_OFF);
    const T* __restrict__ sm_vd = reinterpret_cast<const T*>(st + S::VD_OFF);
    const float* __restrict__ sm_wx = reinterpret_cast<const float*>(st + S::WX_OFF);
    const float* __restrict__ sm_wz = reinterpret_cast<const float*>(st + S::WZ_OFF);

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int nze = d.nze, nb = d.nb, nx = d.nx, lds = d.lds, zs0 = d.zs0;
    const bool first = t.first;
    const bool do_image = t.do_image;

    // A band with few live rows (the last band of a shot) packs several columns
    // into one warp: G = 2^t.glog lanes per column (set by the producer) and
    // 32 / G columns per pass.  Passes go round-robin over the consumer warps
    // (first_item), so that the packed bands of successive tiles land on
    // different warps.  G = 32 is one column per pass.
    const int lg = t.glog;
    const int G = 1 << lg;
    const int cpp = 32 >> lg;
    const int sub = lane & (G - 1);              // this thread's float4 slot in the column
    const int zr = t.z0 + 4 * sub;               // first of this thread's 4 rows
    const bool lane_in = zr < nze;
    const bool lane_snap = lane_in && zr >= zs0 && zr < zs0 + lds;

    const T c0 = (T)d.c0;
    const float* cx = d.cx;     // read from shared memory (as float4s) where used
    const float* cz = d.cz;

    float wz[4];
    {
        const float4 w4 = *reinterpret_cast<const float4*>(sm_wz + 4 * sub);
        wz[0] = w4.x; wz[1] = w4.y; wz[2] = w4.z; wz[3] = w4.w;
    }

    const int npass = TX / cpp;
    const int f = first_item<NCW>(t, TX, warp);
#pragma unroll
    for (int c = 0; c < (TX + NCW - 1) / NCW; ++c) {
        const int ps = f + c * NCW;
        if (ps >= npass) continue;               // warp-uniform
        const int lx = ps * cpp + (lane >> lg);
        const int x = t.x0 + lx;
        const T* col = sm_pc + (lx + H) * S::SZ + 4 * sub + HP;   // row zr of column x
        const bool col_int = (x >= nb) && (x < nb + nx);
        const uint32_t ic = (uint32_t)(x - nb) * (uint32_t)lds + (uint32_t)(zr - zs0);

        // Backward stored steps: start the snapshot and image loads of this
        // column first so their latency overlaps the stencil arithmetic.
        T fs[4], Iv[4], Sv[4];
        if (do_image && lane_snap && col_int) {
            const size_t cell = (size_t)t.ksnap * nx * lds + ic;
            const size_t eidx = ((size_t)t.ksnap * nx + (x - nb)) * d.ntz + t.tz;
            if (psrc)   // reconstruction: the source field at the imaged level
                ldg4(psrc + (uint32_t)x * (uint32_t)ldz + zr, fs, 0);
            else
                load_snapshot4<T>(d, cell, eidx, fs);
            ldg4(reinterpret_cast<const T*>(d.img) + ic, Iv, 0);
            ldg4(reinterpret_cast<const T*>(d.ill) + ic, Sv, 0);
        }

        T pp[4], vd[4];   // pp is stale on a first step, where ColumnMath does not read it
        ld4(sm_vd + lx * kTileZ + 4 * sub, vd);
        ld4(sm_pp + lx * kTileZ + 4 * sub, pp);
        T val[4];
        ColumnMath<T, H, EXACT, S::SZ, HP>::run(col, pp, vd, sm_wx[lx], wz, c0, cx, cz, first, val);
        int rkb = 0, rke = 0;
        if (t.has_pts) {
            const int* __restrict__ off = reinterpret_cast<const int*>(st + (t.rec_staged ? S::RCS_OFF : S::CS_OFF));
            rkb = off[lx];
            rke = off[lx + 1];
        }
        column_epilogue<T, H, EXACT>(d, t, x, zr, lane, lane_in, lane_snap, val, vd, fs, Iv, Sv, rkb, rke,
                                     reinterpret_cast<const RecEntry*>(st + S::REC_OFF), pcur, pnext, ldz, G);
    }
}

// ------------------------------------------------- pipeline control block
// Shared memory of the step kernel: a 128-byte control block, then `nstage`
// stages of TileShape::STAGE bytes each.
//   [0, 32)    full[s]:  completes when the producer warp has written the
//              stage header (all 32 lanes arrive) and the TMA boxes landed
//   [32, 64)   empty[s]: completes when every consumer thread is done with it
//   [64, 68)   abort flag (a bounded wait gave up somewhere in the CTA)
//   [80, 96)   issued[s]: tiles the producer has issued into stage s
constexpr int kMaxStages = 4;
constexpr int kCtrlBytes = 128;

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.expect_tx.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Programmatic dependent launch: wait until the previous grid in the stream
// has completed and its memory is visible, and let the next grid launch early
// (its CTAs then only wait in griddep_wait for this grid to finish).
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void griddep_launch_dependents() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Bounded wait that also gives up as soon as another warp of the CTA aborted.
__device__ __forceinline__ bool mbar_wait_or_abort(uint64_t* bar, uint32_t parity, volatile int* abort_flag,
                                                   int* err) {
    if (mbar_try_wait_sleep(bar, parity, kSleepHintNs)) return true;
    const unsigned long long t0 = global_ns();
    while (!mbar_try_wait_sleep(bar, parity, kSleepHintNs)) {
        if (*abort_flag) return false;
        if (global_ns() - t0 > kWaitNs) {
            atomicOr(err, kErrTmaTimeout);
            *abort_flag = 1;
            return false;
        }
    }
    return true;
}

// What a tile does at global step g (identical in every lane): active,
// forward or backward pass, time index, first step of the pass, which field
// level holds p^n, stored step, receiver work.  rec_staged is filled later.
__device__ __forceinline__ TileInfo decode_tile(const TileRef& tr, long long g) {
    TileInfo ti{};
    const long long n = g - tr.g0;
    ti.active = n >= 0 && n < tr.total_steps;
    if (!ti.active) return ti;
    const int nt = tr.nt;
    ti.fwd = n < nt;
    const int j = ti.fwd ? (int)n : (int)(n - nt);
    ti.it = ti.fwd ? j : nt - 1 - j;
    ti.first = j == 0;
    ti.cur = j & 1;
    ti.x0 = tr.x0;
    ti.z0 = tr.z0;
    ti.tz = tr.z0 / kTileZ;
    const int ks = ti.it / tr.si;
    const bool stored = ks * tr.si == ti.it;
    ti.do_snap = ti.fwd && stored && (tr.flags & kFlagSnapshots);
    ti.do_image = !ti.fwd && stored && (tr.flags & kFlagImage);
    ti.ksnap = ks;
    const bool pts_matter = !ti.fwd || (tr.flags & kFlagRecord);
    ti.has_pts = pts_matter && tr.has_pts;
    ti.prv = ti.cur ^ 1;
    ti.src = -1;
    if (tr.flags & kFlagSourceTile) {
        // The source field run backwards during the backward pass of step it:
        // level L(it) = 2 L(it+1) - L(it+2) + (v dt)^2 lap L(it+1) + injection of
        // wavelet sample it+1, the forward update with the two levels swapped
        // (level m lives in slot buffer m & 1).  L(nt) and L(nt-1) are what the
        // forward pass left; L(0) is never imaged.
        if (ti.fwd || ti.it < 1 || ti.it > nt - 2) {
            ti.active = 0;
            return ti;
        }
        ti.recon = 1;
        ti.fwd = 1;            // injects like a forward step ...
        ti.it = ti.it + 1;     // ... the wavelet sample of level it+1
        ti.cur = ti.it & 1;
        ti.prv = ti.cur ^ 1;
        ti.first = 0;
        ti.do_snap = ti.do_image = 0;
        ti.has_pts = 0;
        return ti;
    }
    if (tr.flags & kFlagRecon) {
        if (ti.fwd) {
            ti.strip = ti.it <= nt - 2;            // level it+1 of the source field
        } else {                                   // receiver field in slot buffers 3, 4
            ti.cur += 3;
            ti.prv += 3;
            ti.src = (ti.it + 1) & 1;              // the source field at level it+1
        }
    }
    return ti;
}

// Stages the receivers of columns [x0, x0 + ncols) into re[] with per-column
// offsets rcs[0..ncols] (warp-cooperative).  Returns false,
// staging nothing, when the columns hold more than kTileRec receivers.  `sd`
// is the stage's copy of the descriptor.  Two dependent rounds of global loads
// (the column offsets, then the receivers' rows, indices and trace samples).
__device__ __forceinline__ bool stage_receivers(const ShotDesc& sd, const TileInfo& ti, int x0, int ncols, int nxe,
                                                int* rcs, RecEntry* re) {
    const int lane = threadIdx.x & 31;
    const int* rec_col = sd.rec_col;
    if (!rec_col) return false;
    // column offsets, clamped to nxe (rec_col has nxe + 1 entries)
    const int xk = x0 + lane < nxe ? x0 + lane : nxe;
    const int xe = x0 + ncols < nxe ? x0 + ncols : nxe;
    const int r_lo = __ldg(rec_col + x0);
    const int nrec = __ldg(rec_col + xe) - r_lo;
    const int ok = __ldg(rec_col + xk);
    if (nrec > kTileRec) return false;
    if (lane <= ncols) rcs[lane] = ok - r_lo;
    for (int k = lane + 32; k <= ncols; k += 32) {
        const int x = x0 + k < nxe ? x0 + k : nxe;
        rcs[k] = __ldg(rec_col + x) - r_lo;
    }
    const int* pts_ir = sd.pts_ir + r_lo;
    const int* rec_zs = sd.rec_zs + r_lo;
    constexpr int kPer = kTileRec / 32;
    int ir[kPer], rz[kPer];
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
        const int k = lane + 32 * u;
        ir[u] = k < nrec ? __ldg(pts_ir + k) : 0;
        rz[u] = k < nrec ? __ldg(rec_zs + k) : 0;
    }
    float tr[kPer];
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
        const int k = lane + 32 * u;
        tr[u] = (k < nrec && !ti.fwd) ? __ldg(sd.traces + (size_t)ir[u] * sd.trace_nt + ti.it) : 0.f;
    }
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
        const int k = lane + 32 * u;
        if (k < nrec) re[k] = RecEntry{rz[u], ir[u], tr[u]};
    }
    return true;
}

// What the producer loads for a tile that does not depend on the step: the
// tile's shot descriptor words, its taper weights.  Loaded for a CTA's first
// tile before griddepcontrol.wait, so that their latency overlaps the previous
// step's tail.
constexpr int kDescWords = (int)(sizeof(ShotDesc) / 4);
constexpr int kDescPerLane = (kDescWords + 31) / 32;
struct TileStatic {
    int dw[kDescPerLane];
    float wxv;
    float4 wzv;
};

template <int TX>
__device__ __forceinline__ void load_tile_static(const StepParams& p, const TileRef& tr, TileStatic& ts) {
    const int lane = threadIdx.x & 31;
    const int* src = reinterpret_cast<const int*>(p.descs + tr.slot);
#pragma unroll
    for (int k = 0; k < kDescPerLane; ++k)
        ts.dw[k] = lane + 32 * k < kDescWords ? __ldg(src + lane + 32 * k) : 0;
    const int xw = tr.x0 + lane;
    ts.wxv = (lane < TX && xw < tr.nxe) ? __ldg(tr.wx + xw) : 0.f;
    ts.wzv = make_float4(0.f, 0.f, 0.f, 0.f);
    if (tr.z0 + 4 * lane < tr.nze) ts.wzv = __ldg(reinterpret_cast<const float4*>(tr.wz + tr.z0 + 4 * lane));
}

// Fills one stage with tile `t` (producer warp, all 32 lanes).  Lane 0 decodes
// what the tile does this step and publishes it as TileInfo; the lanes copy
// the shot descriptor, the tile's taper weights and (for tiles with receiver
// cells) the receivers into the stage; every lane then arrives on the stage's
// full barrier (so each lane releases its own writes), lane 0 with the byte
// count of the TMA boxes it issues.  An active tile always loads (v dt)^2; p^n
// (with halo) and p^{n-1} are skipped on the first step of a pass, where both
// are zero.  An inactive tile (its shot is not running at this global step)
// only publishes TileInfo.
//
// The producer is on the critical path of the pipeline, so its global loads
// are issued in as few dependent rounds as possible: the descriptor words and
// both tapers first (before the TMA issue, so their latency overlaps it), the
// receiver tables after the descriptor has reached shared memory.
template <typename T, int H, int NCW, int TX>
__device__ __forceinline__ void produce_tile(unsigned char* st, uint64_t* full, const CUtensorMap* map_pc,
                                             const CUtensorMap* map_box, const StepParams& p, const TileRef& tr,
                                             long long g, const TileStatic* pre) {
    using S = TileShape<T, H, NCW, TX>;
    static_assert(S::TX <= 32, "one producer lane per tile column");
    static_assert(kTileZ == 4 * 32, "one float4 of the z taper per producer lane");
    static_assert((S::TX & (S::TX - 1)) == 0, "tile width is a power of two");
    const int lane = threadIdx.x & 31;
    TileInfo ti = decode_tile(tr, g);
    if (!ti.active) {
        if (lane == 0) *reinterpret_cast<TileInfo*>(st + S::INFO_OFF) = ti;
        mbar_arrive(full);
        return;
    }
    const int x0 = tr.x0, z0 = tr.z0, nxe = tr.nxe;
    // Lanes per column of the band: the fewest float4 lanes that cover its live
    // rows (a power of two), and at least 32 / TX so that one pass of a warp
    // stays inside the tile.
    {
        const int live = tr.nze - z0 < kTileZ ? tr.nze - z0 : kTileZ;
        const int need = (live + 3) >> 2;
        const int lg = need <= 1 ? 0 : 32 - __clz(need - 1);
        constexpr int kMinLg = 5 - ilog2(S::TX);
        ti.glog = lg > kMinLg ? lg : kMinLg;
    }
    // A plain tile needs none of the epilogue's per-cell tests: it lies inside
    // the ring of H zero cells on every side and holds no source or receiver
    // work this step.
    ti.plain = x0 >= H && x0 + S::TX <= nxe - H && z0 >= H && z0 + kTileZ <= tr.nze - H && !ti.has_pts &&
               !(ti.fwd && tr.has_src) && !ti.recon && !(ti.strip && (tr.flags & kFlagBandTile));

    TileStatic ts;
    if (pre)
        ts = *pre;
    else
        load_tile_static<S::TX>(p, tr, ts);
    const int* dw = ts.dw;
    const int xw = x0 + lane;
    const float wxv = ts.wxv;
    const float4 wzv = ts.wzv;
    // Sponge weight exactly 1 on every live cell of the tile (its live columns
    // and rows): the consumers then skip the weight multiplies.
    {
        const int zl = z0 + 4 * lane;
        const bool xok = lane >= S::TX || xw >= nxe || wxv == 1.0f;
        const bool zok = (zl >= tr.nze || wzv.x == 1.0f) && (zl + 1 >= tr.nze || wzv.y == 1.0f) &&
                         (zl + 2 >= tr.nze || wzv.z == 1.0f) && (zl + 3 >= tr.nze || wzv.w == 1.0f);
        ti.unitw = __all_sync(0xffffffffu, xok && zok) ? 1 : 0;
    }

    if (lane == 0) {
        *reinterpret_cast<TileInfo*>(st + S::INFO_OFF) = ti;
        if (ti.first) {
            mbar_expect_tx(full, S::BOX_BYTES);
        } else {
            mbar_expect_tx(full, S::PC_BYTES + 2 * S::BOX_BYTES);
            tma_load_3d(st + S::PC_OFF, map_pc, full, z0 - S::HP, x0 - H, tr.field_base + ti.cur);
            tma_load_3d(st + S::PP_OFF, map_box, full, z0, x0, tr.field_base + ti.prv);
        }
        tma_load_3d(st + S::VD_OFF, map_box, full, z0, tr.vd_x, tr.vd_buf);
    }
    {
        int* dst = reinterpret_cast<int*>(st + S::DESC_OFF);
#pragma unroll
        for (int k = 0; k < kDescPerLane; ++k)
            if (lane + 32 * k < kDescWords) dst[lane + 32 * k] = dw[k];
    }
    if (lane < S::TX) reinterpret_cast<float*>(st + S::WX_OFF)[lane] = wxv;
    reinterpret_cast<float4*>(st + S::WZ_OFF)[lane] = wzv;
    if (!ti.has_pts && !ti.do_image) {
        mbar_arrive(full);
        return;
    }
    __syncwarp();
    const ShotDesc& sd = *reinterpret_cast<const ShotDesc*>(st + S::DESC_OFF);
    if (ti.has_pts) {
        // Stage the tile's receivers (row, index and, backward, this step's
        // trace sample) so consumers never chase the receiver lists in global
        // memory; a tile with more than kTileRec receivers keeps the global path.
        const bool staged = stage_receivers(sd, ti, x0, S::TX, nxe, reinterpret_cast<int*>(st + S::RCS_OFF),
                                            reinterpret_cast<RecEntry*>(st + S::REC_OFF));
        if (!staged)
            for (int k = lane; k <= S::TX; k += 32) {
                const int x = x0 + k < nxe ? x0 + k : nxe;
                reinterpret_cast<int*>(st + S::CS_OFF)[k] = __ldg(sd.col_start + x);
            }
        if (lane == 0) reinterpret_cast<TileInfo*>(st + S::INFO_OFF)->rec_staged = staged ? 1 : 0;
    }
    // Stored backward steps: pull the tile's snapshot, image and illumination
    // lines (and their compensation words) into L2 now, so that the consumers'
    // loads of them a tile later hit L2 instead of HBM.
    if (ti.do_image) {
        const int zs0 = sd.zs0, lds = sd.lds, nb = sd.nb, nx = sd.nx;
        const int r0 = z0 > zs0 ? z0 : zs0;
        const int r1 = z0 + kTileZ < zs0 + lds ? z0 + kTileZ : zs0 + lds;
        const bool comp = sd.acc_mode != kAccPlain;
        const int snap_es = (sd.snap_type == kSnapF32) ? 4 : (sd.snap_type == kSnapF64 ? 8 : 2);
        if (r1 > r0)
#pragma unroll 1
            for (int a = 0; a < 5; ++a) {
                const char* base =
                    a == 0 ? (ti.src < 0 && sd.snap ? reinterpret_cast<const char*>(sd.snap) +
                                                          (size_t)ti.ksnap * nx * lds * snap_es
                                                    : nullptr)
                    : a == 1 ? reinterpret_cast<const char*>(sd.img)
                    : a == 2 ? reinterpret_cast<const char*>(sd.ill)
                    : a == 3 ? (comp ? reinterpret_cast<const char*>(sd.img_c) : nullptr)
                             : (comp ? reinterpret_cast<const char*>(sd.ill_c) : nullptr);
                const int es = a == 0 ? snap_es : (a >= 3 ? 2 : (int)sizeof(T));   // BF16 compensation words
                if (!base) continue;
                const int lpc = ((r1 - r0) * es + 127) >> 7;
                for (int idx = lane; idx < S::TX * lpc; idx += 32) {
                    const int c = idx / lpc, l = idx - c * lpc;
                    const int xi = x0 + c - nb;
                    if (xi < 0 || xi >= nx) continue;
                    const char* q = base + ((size_t)xi * lds + (r0 - zs0)) * es + (size_t)l * 128;
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(q));
                }
            }
    }
    mbar_arrive(full);
}

// ------------------------------------------------------- per-step kernel
// One launch = one time step of every tile in the tile list.  Persistent and
// warp-specialised: warp NCW is the producer, which walks the CTA's tiles
// (stride gridDim.x) and fills a ring of `nstage` shared-memory stages; warps
// 0..NCW-1 are consumers that compute each tile as soon as its stage is full
// and release it.  No CTA-wide barrier inside the loop: the producer runs up to
// nstage-1 tiles ahead of the consumers, so TMA latency hides behind compute.
//
// The CTAs per SM of each shape (and so its register budget) are those of
// step_ctas_per_sm in kernels.hpp.
template <typename T, int H, bool EXACT, int NCW, int TX>
__global__ void __launch_bounds__((NCW + 1) * 32, sizeof(T) == 8 ? 1 : (NCW == 4 ? 3 : (TX == 16 ? 2 : 1)))
    step_kernel(const __grid_constant__ CUtensorMap map_pc, const __grid_constant__ CUtensorMap map_box,
                const StepParams p) {
    using S = TileShape<T, H, NCW, TX>;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw);
    uint64_t* empty = full + kMaxStages;
    volatile int* abort_flag = reinterpret_cast<volatile int*>(smem_raw + 64);
    int* issued = reinterpret_cast<int*>(smem_raw + 80);
    unsigned char* stages = smem_raw + kCtrlBytes;
    const int nst = p.nstage;

    if ((int)blockIdx.x >= p.ntiles) return;
    if (threadIdx.x == 0) {
        for (int s = 0; s < nst; ++s) {
            mbar_init(full + s, 32);
            mbar_init(empty + s, NCW * 32);
            issued[s] = 0;
        }
        *abort_flag = 0;
        fence_mbar_init();
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5;
    // The producer's first tile: its reference, descriptor and tapers do not
    // depend on the previous step, so they load before the wait below.
    TileRef cur{};
    TileStatic first{};
    if (warp == NCW) {
        cur = p.tiles[blockIdx.x];
        load_tile_static<S::TX>(p, cur, first);
    }
    griddep_wait();
    griddep_launch_dependents();
    const long long g = *p.step_counter + p.step_offset;

    if (warp == NCW) {
        int s = 0, round = 0;   // stage and how many times the ring has wrapped
        TileRef nxt = cur;
        for (int t = blockIdx.x; t < p.ntiles; t += gridDim.x) {
            if (t + (int)gridDim.x < p.ntiles) nxt = p.tiles[t + gridDim.x];   // in flight while we wait
            if (round > 0 && !mbar_wait_or_abort(empty + s, (round - 1) & 1, abort_flag, p.error_word)) break;
            // Failure-detection test: a tile whose stage is never filled makes the
            // consumers' bounded wait run out (no copy is in flight for it).
            if (t != p.stall_tile) {
                produce_tile<T, H, NCW, TX>(stages + (size_t)s * S::STAGE, full + s, &map_pc, &map_box, p, cur,
                                                g, t == (int)blockIdx.x ? &first : nullptr);
                if ((threadIdx.x & 31) == 0) issued[s] = round + 1;
            }
            cur = nxt;
            if (++s == nst) { s = 0; ++round; }
        }
    } else {
        int s = 0;
        uint32_t phase = 0;   // parity of the current round of the ring
        for (int t = blockIdx.x; t < p.ntiles; t += gridDim.x) {
            const unsigned char* st = stages + (size_t)s * S::STAGE;
            if (!mbar_wait_or_abort(full + s, phase, abort_flag, p.error_word)) break;
            const TileInfo info = *reinterpret_cast<const TileInfo*>(st + S::INFO_OFF);
            if (info.active) {
                const ShotDesc& d = *reinterpret_cast<const ShotDesc*>(st + S::DESC_OFF);
                T* base = reinterpret_cast<T*>(p.fields) + (size_t)d.field_slot * p.slot_stride;
                compute_tile<T, H, EXACT, NCW, TX>(st, info, base + (size_t)info.cur * p.buf_stride,
                                                       base + (size_t)info.prv * p.buf_stride,
                                                       info.src >= 0 ? base + (size_t)info.src * p.buf_stride
                                                                     : nullptr,
                                                       p.ldz);
            }
            mbar_arrive(empty + s);
            if (++s == nst) { s = 0; phase ^= 1u; }
        }
    }
    __syncthreads();
    // After an abort, copies the producer issued may still be in flight: wait
    // (bounded) for the last phase of every stage before the CTA's shared
    // memory goes away.
    if (*abort_flag && threadIdx.x == 0) {
        for (int s = 0; s < nst; ++s)
            if (issued[s] > 0)
                mbar_wait_bounded(full + s, (uint32_t)((issued[s] - 1) & 1), p.error_word, kWaitNs / 4);
    }
}

// Advances the global step counter of a chunk (the last node of a captured
// chunk of step launches).
__global__ void advance_counter_kernel(long long* counter, int by);

}  // namespace rtmb
