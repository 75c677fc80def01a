// march_kernel.cuh -- the register-march variant of the fused leapfrog step.
//
// Same arithmetic, same tile list semantics and the same per-column epilogue
// as step_kernel (step_kernel.cuh), organised for fewer instructions per cell:
//
//   * one warp owns a strip of 128 rows (32 lanes x a float4 of depth cells)
//     by L columns of one shot and marches along x through it;
//   * the 2H+1 columns x-H .. x+H of p^n live in a rotating register queue, so
//     every p^n column is loaded from global memory (L2) once per strip instead
//     of 2H+1 times from shared memory;
//   * the depth neighbours come from the neighbouring lanes by warp shuffles;
//     only the lanes at the strip's top and bottom load the H-row halo;
//   * the next column's p^n, p^{n-1}, (v dt)^2, halo and x-taper are loaded one
//     column ahead, so their latency hides behind the current column's math.
//
// No shared-memory ring, no barriers: a warp's work depends only on the
// previous step, which the launch order (programmatic dependent launches,
// griddepcontrol.wait) guarantees complete.  FP32 only (the register queue of
// an FP64 strip does not fit); FP64 runs on step_kernel.
#pragma once

#include "step_kernel.cuh"

namespace rtmb {

constexpr int kMarchWarps = 4;                 // independent warps per CTA
constexpr int kMarchThreads = kMarchWarps * 32;

// Per-warp shared memory: the item's descriptor and its staged receivers.
struct MarchWarpSmem {
    alignas(16) unsigned char desc[448];
    int rcs[128];                              // per-column receiver offsets (L+1 <= 128)
    RecEntry re[kTileRec];
};

__device__ __forceinline__ float4 ld_f4(const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); }
__device__ __forceinline__ void to4(const float4& v, float (&r)[4]) {
    r[0] = v.x; r[1] = v.y; r[2] = v.z; r[3] = v.w;
}

template <int H, bool EXACT>
__global__ void __launch_bounds__(kMarchThreads) march_kernel(const StepParams p) {
    using T = float;
    using A = Arith<T, EXACT>;
    constexpr int R = 2 * H + 1;
    constexpr int HP = Halo<H>::HP;
    __shared__ MarchWarpSmem wsm[kMarchWarps];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    MarchWarpSmem& W = wsm[warp];

    griddep_wait();
    griddep_launch_dependents();
    const long long g = *p.step_counter + p.step_offset;
    const int ldz = p.ldz;
    const int M = p.march_m;
    const int L = R * M;

    for (int t = blockIdx.x * kMarchWarps + warp; t < p.ntiles; t += gridDim.x * kMarchWarps) {
        const TileRef tr = p.tiles[t];
        TileInfo ti = decode_tile(tr, g);
        if (!ti.active) continue;
        __syncwarp();   // the previous item is done with this warp's shared memory
        {
            const int* src = reinterpret_cast<const int*>(p.descs + tr.slot);
            int* dst = reinterpret_cast<int*>(W.desc);
            for (int i = lane; i < (int)(sizeof(ShotDesc) / 4); i += 32) dst[i] = __ldg(src + i);
        }
        const ShotDesc& gd = p.descs[tr.slot];
        const int nxe = tr.nxe, nze = tr.nze, x0 = tr.x0, z0 = tr.z0;
        ti.rec_staged = 0;
        if (ti.has_pts) ti.rec_staged = stage_receivers(gd, ti, x0, L, nxe, W.rcs, W.re) ? 1 : 0;
        __syncwarp();
        const ShotDesc& d = *reinterpret_cast<const ShotDesc*>(W.desc);

        T* base = reinterpret_cast<T*>(p.fields) + (size_t)(tr.field_base / p.nbuf) * p.slot_stride;
        T* pc_buf = base + (size_t)ti.cur * p.buf_stride;          // p^n
        T* pn_buf = base + (size_t)(ti.cur ^ 1) * p.buf_stride;    // p^{n-1} in, p^{n+1} out
        const T* vd_buf = base + 2 * (size_t)p.buf_stride;         // (v dt)^2
        const int zr = z0 + 4 * lane;
        const bool lane_rows = zr < ldz;
        const bool lane_in = zr < nze;
        const bool lane_snap = lane_in && zr >= d.zs0 && zr < d.zs0 + d.lds;
        const bool first = ti.first;
        const bool top_ok = z0 > 0;                 // rows z0-HP .. z0-1 exist
        const bool bot_ok = z0 + kTileZ < ldz;      // rows z0+128 .. z0+128+HP-1 exist
        float wz[4] = {0.f, 0.f, 0.f, 0.f};
        if (lane_in) to4(ld_f4(tr.wz + zr), wz);
        const T c0 = (T)d.c0;
        T cx[H + 1], cz[H + 1];
#pragma unroll
        for (int k = 1; k <= H; ++k) {
            cx[k] = (T)d.cx[k];
            cz[k] = (T)d.cz[k];
        }

        auto ldcol = [&](const T* buf, int x, T (&r)[4]) {
            if (x >= 0 && x < nxe && lane_rows) {
                to4(ld_f4(buf + (size_t)x * ldz + zr), r);
            } else {
                r[0] = r[1] = r[2] = r[3] = (T)0;
            }
        };
        // Halo rows of column x for the strip's edge lanes: ht0/ht1 above,
        // hb0/hb1 below (see the zz assembly below for which lane needs what).
        auto ldhalo = [&](int x, T (&ht0)[4], T (&ht1)[4], T (&hb0)[4], T (&hb1)[4]) {
#pragma unroll
            for (int q = 0; q < 4; ++q) ht0[q] = ht1[q] = hb0[q] = hb1[q] = (T)0;
            if (x < 0 || x >= nxe || first) return;
            const T* col = pc_buf + (size_t)x * ldz;
            if (HP == 4) {
                if (lane == 0 && top_ok) to4(ld_f4(col + z0 - 4), ht0);
                if (lane == 31 && bot_ok) to4(ld_f4(col + z0 + kTileZ), hb0);
            } else {
                if (lane == 0 && top_ok) {
                    to4(ld_f4(col + z0 - 8), ht0);
                    to4(ld_f4(col + z0 - 4), ht1);
                }
                if (lane == 1 && top_ok) to4(ld_f4(col + z0 - 4), ht0);
                if (lane == 31 && bot_ok) {
                    to4(ld_f4(col + z0 + kTileZ), hb0);
                    to4(ld_f4(col + z0 + kTileZ + 4), hb1);
                }
                if (lane == 30 && bot_ok) to4(ld_f4(col + z0 + kTileZ), hb0);
            }
        };

        // Queue: column x0-H+j lives in slot j % R.  Preload x0-H .. x0+H-1.
        T q[R][4];
#pragma unroll
        for (int j = 0; j < R; ++j) q[j][0] = q[j][1] = q[j][2] = q[j][3] = (T)0;
        if (!first) {
#pragma unroll
            for (int j = 0; j < 2 * H; ++j) ldcol(pc_buf, x0 - H + j, q[j]);
        }
        // Loads for the first column (prefetched one column ahead from then on).
        T lead[4] = {0, 0, 0, 0}, ppn[4] = {0, 0, 0, 0}, vdn[4];
        T ht0n[4], ht1n[4], hb0n[4], hb1n[4];
        if (!first) {
            ldcol(pc_buf, x0 + H, lead);
            ldcol(pn_buf, x0, ppn);
        }
        ldcol(vd_buf, x0, vdn);
        ldhalo(x0, ht0n, ht1n, hb0n, hb1n);
        float wxn = x0 < nxe ? __ldg(tr.wx + x0) : 0.f;

        for (int b = 0; b < M; ++b) {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int c = b * R + r;
                const int x = x0 + c;
                // this column's inputs (loaded during the previous column)
#pragma unroll
                for (int k = 0; k < 4; ++k) q[(r + 2 * H) % R][k] = lead[k];
                T pp[4], vd[4], ht0[4], ht1[4], hb0[4], hb1[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    pp[k] = ppn[k]; vd[k] = vdn[k];
                    ht0[k] = ht0n[k]; ht1[k] = ht1n[k]; hb0[k] = hb0n[k]; hb1[k] = hb1n[k];
                }
                const float wxv = wxn;
                // next column's inputs
                if (c + 1 < L) {
                    if (!first) {
                        ldcol(pc_buf, x + 1 + H, lead);
                        ldcol(pn_buf, x + 1, ppn);
                    }
                    ldcol(vd_buf, x + 1, vdn);
                    ldhalo(x + 1, ht0n, ht1n, hb0n, hb1n);
                    wxn = x + 1 < nxe ? __ldg(tr.wx + x + 1) : 0.f;
                }
                // stored backward steps: snapshot and image loads of this column
                const bool col_int = (x >= d.nb) && (x < d.nb + d.nx);
                T fs[4], Iv[4], Sv[4];
                if (ti.do_image && lane_snap && col_int) {
                    const uint32_t ic = (uint32_t)(x - d.nb) * (uint32_t)d.lds + (uint32_t)(zr - d.zs0);
                    const size_t cell = (size_t)ti.ksnap * d.nx * d.lds + ic;
                    const size_t eidx = ((size_t)ti.ksnap * d.nx + (x - d.nb)) * d.ntz + ti.tz;
                    load_snapshot4<T>(d, cell, eidx, fs);
                    ldg4(reinterpret_cast<const T*>(d.img) + ic, Iv, 0);
                    ldg4(reinterpret_cast<const T*>(d.ill) + ic, Sv, 0);
                }
                // depth neighbours of the centre column
                const T* ctr = q[(r + H) % R];
                T zz[4 + 2 * HP];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    zz[HP + k] = ctr[k];
                    const T up1 = __shfl_up_sync(0xffffffffu, ctr[k], 1);
                    const T dn1 = __shfl_down_sync(0xffffffffu, ctr[k], 1);
                    if (HP == 4) {
                        zz[k] = lane == 0 ? ht0[k] : up1;
                        zz[HP + 4 + k] = lane == 31 ? hb0[k] : dn1;
                    } else {
                        const T up2 = __shfl_up_sync(0xffffffffu, ctr[k], 2);
                        const T dn2 = __shfl_down_sync(0xffffffffu, ctr[k], 2);
                        zz[k] = lane <= 1 ? ht0[k] : up2;
                        zz[4 + k] = lane == 0 ? ht1[k] : up1;
                        zz[HP + 4 + k] = lane == 31 ? hb0[k] : dn1;
                        zz[HP + 8 + k] = lane == 31 ? hb1[k] : (lane == 30 ? hb0[k] : dn2);
                    }
                }
                // the stencil, in the reference's operation order
                T lap[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) lap[k] = A::mul(c0, zz[HP + k]);
#pragma unroll
                for (int k = 1; k <= H; ++k) {
                    const T* xm = q[(r + H - k) % R];
                    const T* xp = q[(r + H + k) % R];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const T ax = A::add(xp[u], xm[u]);
                        const T az = A::add(zz[HP + u + k], zz[HP + u - k]);
                        lap[u] = A::add(lap[u], A::add(A::mul(cx[k], ax), A::mul(cz[k], az)));
                    }
                }
                T val[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const T w = (T)__fmul_rn(wxv, wz[u]);
                    const T prev = A::mul(pp[u], w);
                    const T s = A::add(A::sub(A::mul((T)2, zz[HP + u]), prev), A::mul(vd[u], lap[u]));
                    val[u] = A::mul(s, w);
                }
                int rkb = 0, rke = 0;
                if (ti.has_pts) {
                    if (ti.rec_staged) {
                        rkb = W.rcs[c];
                        rke = W.rcs[c + 1];
                    } else if (x < nxe) {
                        rkb = __ldg(d.col_start + x);
                        rke = __ldg(d.col_start + x + 1);
                    }
                }
                column_epilogue<T, H, EXACT>(d, ti, x, zr, lane, lane_in, lane_snap, val, vd, fs, Iv, Sv, rkb, rke,
                                             W.re, pc_buf, pn_buf, ldz, 32);
            }
        }
    }
}

}  // namespace rtmb
