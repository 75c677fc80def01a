// step_kernel.cuh -- the fused leapfrog time step for sm_100a.
//
// One CTA advances one 128-row x TX-column tile of one shot by one time step.
// What the reference does in five passes per step (fd_time_step, inject_*,
// apply_sponge, save_snapshot / imaging; reference src/rtm/forward.cpp:29-125,
// backward.cpp:20-75, imaging.cpp:25-40) happens here in one:
//
//   1. one elected thread issues a 3D TMA tile load of p^n (tile + stencil halo)
//      from HBM/L2 into shared memory, while every thread prefetches its own
//      p^{n-1}, (v dt)^2 and taper values with 16-byte vector loads;
//   2. each thread owns 4 consecutive depth cells (a float4) of COLS columns and
//      evaluates the order-2H Laplacian from shared memory;
//   3. p^{n+1} = w (2 p^n - w p^{n-1} + vdt2 lap) + injection, written in place
//      over p^{n-1} (only the owning thread touches that cell, so two time
//      levels suffice and there is no read/write race);
//   4. on stored steps the forward pass writes the interior snapshot (FP32, or
//      BF16/FP16 with a power-of-two scale per 128-cell column segment) and the
//      backward pass correlates with the stored snapshot (I += f b, S += f^2),
//      either straight into the running image or into per-shot compensated sums.
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

// 2^e as a float, exact for e in [-126, 127].
__device__ __forceinline__ float pow2f(int e) { return __int_as_float((e + 127) << 23); }

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
// Plain (non-multicast) tiled TMA load of a 3D box from this GPU's own memory.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1,
                                            int c2) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_addr(bar)), "r"(c0), "r"(c1), "r"(c2)
        : "memory");
}

// Bounded wait: gives up after `limit` polls and reports it in the error word.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int* err, long long limit) {
    long long n = 0;
    while (!mbar_try_wait(bar, parity)) {
        if (++n > limit) {
            atomicOr(err, kErrTmaTimeout);
            return false;
        }
    }
    return true;
}

constexpr long long kWaitLimit = 1ll << 22;

// Halo depth in rows, rounded up to 4 so the TMA box starts 16-byte aligned.
template <int H>
struct Halo {
    static constexpr int HP = (H + 3) & ~3;
};

template <typename T, int H, int NWARP, int COLS>
struct TileShape {
    static constexpr int HP = Halo<H>::HP;
    static constexpr int TX = NWARP * COLS;
    static constexpr int SZ = kTileZ + 2 * HP;   // rows held in shared memory
    static constexpr int SX = TX + 2 * H;        // columns held in shared memory
    static constexpr int BYTES = SZ * SX * (int)sizeof(T);
    static constexpr int DESC_BYTES = 512;                      // barrier + staged ShotDesc
    static constexpr int SMEM = DESC_BYTES + ((BYTES + 127) & ~127);
};

// ------------------------------------------------------------- the tile
// Computes one tile after its p^n box has landed in shared memory.
template <typename T, int H, bool EXACT, int NWARP, int COLS>
__device__ __forceinline__ void compute_tile(const ShotDesc& d, const T* __restrict__ sm, T* __restrict__ pcur,
                                             T* __restrict__ pnext, int ldz, int x0, int z0, int tz, int it,
                                             bool fwd, bool first) {
    using A = Arith<T, EXACT>;
    using S = TileShape<T, H, NWARP, COLS>;
    constexpr int HP = S::HP;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int zr = z0 + 4 * lane;                // first of this thread's 4 rows
    const bool lane_in = zr < d.nze;
    const int nxe = d.nxe, nze = d.nze;

    const T c0 = (T)d.c0;
    T cx[H + 1], cz[H + 1];
#pragma unroll
    for (int k = 1; k <= H; ++k) { cx[k] = (T)d.cx[k]; cz[k] = (T)d.cz[k]; }

    // Row masks: rows inside [H, nze-H) are updated, the outer H-ring stays 0.
    bool row_ok[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) row_ok[q] = (zr + q >= H) && (zr + q < nze - H);

    float wzv[4] = {0.f, 0.f, 0.f, 0.f};
    if (lane_in) ldg4(d.wz + zr, wzv);

    const bool store_step = (it % d.si) == 0;
    const bool do_snap = fwd && store_step && (d.flags & kFlagSnapshots);
    const bool do_image = !fwd && store_step && (d.flags & kFlagImage);
    const int ksnap = it / d.si;
    const bool lane_snap = lane_in && zr >= d.zs0 && zr < d.zs0 + d.lds;

#pragma unroll 1
    for (int c = 0; c < COLS; ++c) {
        const int x = x0 + warp * COLS + c;
        if (x >= nxe) break;                     // warp-uniform
        const int sx = x - x0 + H;               // column inside the smem tile
        const T* col = sm + (size_t)sx * S::SZ + 4 * lane + HP;   // row zr in smem

        // p^{n-1} (own cells), vdt2 (model column clamped to the window), taper
        T pp[4] = {0, 0, 0, 0};
        float vd[4] = {0.f, 0.f, 0.f, 0.f};
        T* pn_col = pnext + (size_t)x * ldz;
        if (lane_in) {
            if (!first) ld4(pn_col + zr, pp);
            int mx = x - d.nb;
            mx = mx < 0 ? 0 : (mx > d.win_nx - 1 ? d.win_nx - 1 : mx);
            ldg4(d.vdt2 + (size_t)(mx + d.model_x0) * d.ldz_model + zr, vd);
        }
        const float wxv = __ldg(d.wx + x);

        // Laplacian from shared memory (zero on the first step of a pass).
        T zz[4 + 2 * HP];
        T lap[4], pc[4];
        if (!first) {
#pragma unroll
            for (int g = 0; g < (4 + 2 * HP) / 4; ++g) {
                T t[4];
                ld4(col - HP + 4 * g, t);
#pragma unroll
                for (int q = 0; q < 4; ++q) zz[4 * g + q] = t[q];
            }
        } else {
#pragma unroll
            for (int i = 0; i < 4 + 2 * HP; ++i) zz[i] = (T)0;
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            pc[q] = zz[HP + q];
            lap[q] = A::mul(c0, pc[q]);
        }
#pragma unroll
        for (int k = 1; k <= H; ++k) {
            T xm[4], xp[4];
            if (!first) {
                ld4(col - (size_t)k * S::SZ, xm);
                ld4(col + (size_t)k * S::SZ, xp);
            } else {
#pragma unroll
                for (int q = 0; q < 4; ++q) { xm[q] = (T)0; xp[q] = (T)0; }
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const T ax = A::add(xp[q], xm[q]);
                const T az = A::add(zz[HP + q + k], zz[HP + q - k]);
                lap[q] = A::add(lap[q], A::add(A::mul(cx[k], ax), A::mul(cz[k], az)));
            }
        }

        // Leapfrog with the sponge folded in.
        const bool col_ok = (x >= H) && (x < nxe - H);
        T val[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const T w = (T)__fmul_rn(wxv, wzv[q]);
            const T prev = A::mul(pp[q], w);
            const T s = A::add(A::sub(A::mul((T)2, pc[q]), prev), A::mul((T)vd[q], lap[q]));
            val[q] = (col_ok && row_ok[q]) ? A::mul(s, w) : (T)0;
        }

        // Injection: the source (forward) or the receivers (backward) at cells
        // whose taper is exactly 1, so adding after the damping matches the
        // reference's inject-then-damp order bit for bit.
        if (fwd) {
            if (x == d.src_x) {
                const T amp = (T)__ldg(d.wavelet + it);
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    if (zr + q == d.src_z) val[q] = A::add(val[q], A::mul((T)vd[q], amp));
            }
        }
        // Receiver cells of this column: inject (backward) or record (forward
        // modelling).  Several receivers on one cell add in ascending ir order,
        // like the reference's sequential loop (backward.cpp:20-27).
        const bool rec_fwd = fwd && (d.flags & kFlagRecord);
        if (!fwd || rec_fwd) {
            const int pb = __ldg(d.col_start + x), pe = __ldg(d.col_start + x + 1);
            for (int j = pb; j < pe; ++j) {
                const PointEntry e = d.pts[j];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    if (e.z != zr + q) continue;
                    for (int r = 0; r < e.ir_count; ++r) {
                        const int ir = __ldg(d.pts_ir + e.ir_begin + r);
                        if (rec_fwd) {
                            d.rec_out[(size_t)ir * d.nt + it] = (float)val[q];
                        } else {
                            const T tr = (T)__ldg(d.traces + (size_t)ir * d.trace_nt + it);
                            val[q] = A::add(val[q], A::mul((T)vd[q], tr));
                        }
                    }
                }
            }
        }

        if (lane_in) {
            st4(pn_col + zr, val);
            if (first) {   // p^n of the first step is zero: clear the other level too
                const T z4[4] = {0, 0, 0, 0};
                st4(pcur + (size_t)x * ldz + zr, z4);
            }
        }

        const bool col_int = (x >= d.nb) && (x < d.nb + d.nx);
        if (col_int && (do_snap || do_image)) {
            const size_t cell = ((size_t)ksnap * d.nx + (x - d.nb)) * d.lds + (zr - d.zs0);
            const size_t eidx = ((size_t)ksnap * d.nx + (x - d.nb)) * d.ntz + tz;
            if (do_snap) {
                if (d.snap_type == kSnapF32 || d.snap_type == kSnapF64) {
                    if (lane_snap) st4cs(reinterpret_cast<T*>(d.snap) + cell, val);
                } else {
                    // power-of-two scale per (snapshot, column, 128-row segment)
                    float amax = 0.f;
                    if (lane_snap)
#pragma unroll
                        for (int q = 0; q < 4; ++q) amax = fmaxf(amax, fabsf((float)val[q]));
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) amax = fmaxf(amax, __shfl_xor_sync(0xffffffffu, amax, o));
                    int e = 0;
                    if (amax > 0.f) {
                        frexpf(amax, &e);          // amax <= 2^e
                        e -= 15;                   // scaled max <= 2^15
                        e = e < -126 ? -126 : (e > 127 ? 127 : e);
                    }
                    if (lane == 0) d.snap_exp[eidx] = (int8_t)e;
                    if (lane_snap) {
                        const float inv = pow2f(-e);
                        uint2 packed;
                        if (d.snap_type == kSnapF16) {
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
                        __stcs(reinterpret_cast<uint2*>(reinterpret_cast<uint16_t*>(d.snap) + cell), packed);
                    }
                }
            }
            if (do_image && lane_snap) {
                T f[4];
                if (d.snap_type == kSnapF32 || d.snap_type == kSnapF64) {
                    ld4cs(reinterpret_cast<const T*>(d.snap) + cell, f);
                } else {
                    const uint2 packed = __ldcs(reinterpret_cast<const uint2*>(
                        reinterpret_cast<const uint16_t*>(d.snap) + cell));
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
                const size_t icell = (size_t)(x - d.nb) * d.lds + (zr - d.zs0);
                T* img = reinterpret_cast<T*>(d.img) + icell;
                T* ill = reinterpret_cast<T*>(d.ill) + icell;
                T I[4], Sv[4];
                ld4(img, I);
                ld4(ill, Sv);
                if (d.acc_mode == kAccPlain) {
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        I[q] = A::add(I[q], A::mul(f[q], val[q]));
                        Sv[q] = A::add(Sv[q], A::mul(f[q], f[q]));
                    }
                } else {
                    // Kahan: sum + (term - comp), comp tracks the lost low part.
                    T* imc = reinterpret_cast<T*>(d.img_c) + icell;
                    T* ilc = reinterpret_cast<T*>(d.ill_c) + icell;
                    T Ic[4], Sc[4];
                    ld4(imc, Ic);
                    ld4(ilc, Sc);
                    using E = Arith<T, true>;
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const T yi = E::sub(E::mul(f[q], val[q]), Ic[q]);
                        const T ti = E::add(I[q], yi);
                        Ic[q] = E::sub(E::sub(ti, I[q]), yi);
                        I[q] = ti;
                        const T ys = E::sub(E::mul(f[q], f[q]), Sc[q]);
                        const T ts = E::add(Sv[q], ys);
                        Sc[q] = E::sub(E::sub(ts, Sv[q]), ys);
                        Sv[q] = ts;
                    }
                    st4(imc, Ic);
                    st4(ilc, Sc);
                }
                st4(img, I);
                st4(ill, Sv);
            }
        }
    }
}

// ------------------------------------------------------- per-step kernel
// One launch = one time step of every tile in the tile list.
template <typename T, int H, bool EXACT, int NWARP, int COLS>
__global__ void __launch_bounds__(NWARP * 32, 3)
    step_kernel(const __grid_constant__ CUtensorMap tmap, const StepParams p) {
    using S = TileShape<T, H, NWARP, COLS>;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw);
    ShotDesc* sd = reinterpret_cast<ShotDesc*>(smem_raw + 16);
    T* tile = reinterpret_cast<T*>(smem_raw + S::DESC_BYTES);

    if ((int)blockIdx.x >= p.ntiles) return;
    const TileRef tr = p.tiles[blockIdx.x];
    {   // stage the shot descriptor in shared memory (read by every thread)
        const int* src = reinterpret_cast<const int*>(p.descs + tr.slot);
        int* dst = reinterpret_cast<int*>(sd);
        for (int i = threadIdx.x; i < (int)(sizeof(ShotDesc) / 4); i += blockDim.x) dst[i] = src[i];
        if (threadIdx.x == 0) {
            mbar_init(bar, 1);
            fence_mbar_init();
        }
        __syncthreads();
    }
    const ShotDesc& d = *sd;
    const long long n = *p.step_counter + p.step_offset - d.g0;
    if (n < 0 || n >= d.total_steps) return;   // shot idle this step
    const bool fwd = n < d.nt;
    const int j = fwd ? (int)n : (int)(n - d.nt);
    const int it = fwd ? j : d.nt - 1 - j;
    const bool first = (j == 0);
    const int cur = j & 1;

    T* base = reinterpret_cast<T*>(p.fields) + (size_t)d.field_slot * p.slot_stride;
    T* pcur = base + (size_t)cur * p.buf_stride;
    T* pnext = base + (size_t)(cur ^ 1) * p.buf_stride;
    const int x0 = tr.tx * S::TX, z0 = tr.tz * kTileZ;

    if (!first) {
        if (threadIdx.x == 0) {
            mbar_arrive_expect_tx(bar, S::BYTES);
            tma_load_3d(tile, &tmap, bar, z0 - S::HP, x0 - H, d.field_slot * 2 + cur);
        }
        if (!mbar_wait_bounded(bar, 0, p.error_word, kWaitLimit)) return;
    }
    compute_tile<T, H, EXACT, NWARP, COLS>(d, tile, pcur, pnext, p.ldz, x0, z0, tr.tz, it, fwd, first);
}

// Advances the global step counter of a chunk (the last node of a captured
// chunk of step launches).
__global__ void advance_counter_kernel(long long* counter, int by);

}  // namespace rtmb
