// rtm_oracle.cpp -- CPU oracle for the 2D acoustic RTM hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file restates, in plain loops, the algorithm
// of the reference CPU engine (Marouane-Djabri/RTM-Acceleration, class
// CPUReferenceRTM) so that the CUDA engine can be checked against it.  The
// product library never links, loads or calls it.
//
// Pinning: the float instance is compared bit-for-bit with images and traces
// produced by the reference's own binaries (compiled by oracle/Makefile into
// oracle/_ref/) and with the SHA-256 the reference records for its Marmousi shot
// file (data/real/marmousi_dataset.sha256:1).  See tests/test_oracle_golden.py.
//
// Every function cites the reference file:line whose behaviour it restates.
// Compile with -ffp-contract=off: the reference's -O2 x86-64 build has no FMA,
// and the float oracle must round exactly like it.
#include "rtm_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <vector>

#include <omp.h>

namespace {

// Taylor central second-derivative weights, orders 2..12
// (reference src/rtm/rtm.cpp:14-23).  Each entry is the correctly rounded float
// of an exact rational, written here as num/den; the reference's table holds
// the same rationals.
struct Rational { double num, den; };
const Rational kCoef[6][7] = {
    {{-2, 1}, {1, 1}},
    {{-5, 2}, {4, 3}, {-1, 12}},
    {{-49, 18}, {3, 2}, {-3, 20}, {1, 90}},
    {{-205, 72}, {8, 5}, {-1, 5}, {8, 315}, {-1, 560}},
    {{-5269, 1800}, {5, 3}, {-5, 21}, {5, 126}, {-5, 1008}, {1, 3150}},
    {{-5369, 1800}, {12, 7}, {-15, 56}, {10, 189}, {-1, 112}, {2, 1925}, {-1, 16632}},
};

// Returns half (order/2) or -1 for an unsupported order (reference rtm.cpp:25-41).
int coefficients(int order, float* c) {
    if (order < 2 || order > 12 || (order & 1)) return -1;
    const int h = order / 2;
    for (int k = 0; k <= h; ++k)
        c[k] = (float)kCoef[h - 1][k].num / (float)kCoef[h - 1][k].den;
    return h;
}

// Reference rtm.cpp:52-55: a = pi^2 f0^2 t^2 evaluated left to right in float.
float ricker_f(float t, float f0) {
    const float a = (float)(M_PI * M_PI) * f0 * f0 * t * t;
    return (1.0f - 2.0f * a) * std::exp(-a);
}

// Everything the time loop needs for one model, in arithmetic type T.
// Tables are built in float exactly like reference rtm_cpu.cpp:9-88 and widened.
template <typename T>
struct Problem {
    int nx = 0, nz = 0, nb = 0, h = 0, nxe = 0, nze = 0, nt = 0, si = 1, nsnap = 0;
    int nthreads = 1;     // host threads for the per-step loops (grids >= 64k cells)
    float dx = 0, dz = 0, ox = 0, oz = 0;
    T c0 = 0, cx[7] = {}, cz[7] = {};
    std::vector<T> vdt2, sponge, wavelet;
    std::vector<T> pp, pc, pn;

    size_t next() const { return (size_t)nxe * nze; }
    size_t nint() const { return (size_t)nx * nz; }
    size_t e(int ixe, int ize) const { return (size_t)ixe * nze + ize; }

    // Reference rtm_cpu.cpp:9-88 (validation :17-22).
    int setup(const oracle_params& p, const float* vel) {
        float c[7];
        h = coefficients(p.order, c);
        if (h < 0) return -1;
        if (p.nb < h + 1) return -2;
        if (p.store_interval < 1) return -3;
        if (p.nx <= 0 || p.nz <= 0 || p.nt <= 0) return -4;
        nx = p.nx; nz = p.nz; nb = p.nb; nt = p.nt; si = p.store_interval;
        dx = p.dx; dz = p.dz; ox = p.ox; oz = p.oz;
        nxe = nx + 2 * nb; nze = nz + 2 * nb;
        nsnap = (nt - 1) / si + 1;

        // v^2 dt^2 on the extended grid, pad cells copy the nearest edge cell.
        const float dt2 = p.dt * p.dt;
        vdt2.assign(next(), 0);
        for (int ixe = 0; ixe < nxe; ++ixe) {
            const int ix = std::min(std::max(ixe - nb, 0), nx - 1);
            for (int ize = 0; ize < nze; ++ize) {
                const int iz = std::min(std::max(ize - nb, 0), nz - 1);
                const float v = vel[(size_t)ix * nz + iz];
                vdt2[e(ixe, ize)] = (T)(v * v * dt2);
            }
        }
        // Cerjan taper exp(-(alpha (nb-d))^2) within nb cells of an edge; the
        // 2D weight is the float product of the two 1D tapers.
        auto taper = [&](int i, int n) -> float {
            const int d = std::min(i, n - 1 - i);
            if (d >= nb) return 1.0f;
            const float a = p.sponge_alpha * (float)(nb - d);
            return std::exp(-a * a);
        };
        std::vector<float> wx(nxe), wz(nze);
        for (int i = 0; i < nxe; ++i) wx[i] = taper(i, nxe);
        for (int i = 0; i < nze; ++i) wz[i] = taper(i, nze);
        sponge.assign(next(), 1);
        for (int ixe = 0; ixe < nxe; ++ixe)
            for (int ize = 0; ize < nze; ++ize)
                sponge[e(ixe, ize)] = (T)(wx[ixe] * wz[ize]);
        // Ricker delayed by 1.2/f0.
        wavelet.resize(nt);
        const float t0 = 1.2f / p.f0;
        for (int it = 0; it < nt; ++it)
            wavelet[it] = (T)ricker_f((float)it * p.dt - t0, p.f0);
        // Coefficients divided by the spacing, in float, then widened.
        const float idx2 = 1.0f / (dx * dx), idz2 = 1.0f / (dz * dz);
        c0 = (T)(c[0] * (idx2 + idz2));
        for (int k = 1; k <= h; ++k) { cx[k] = (T)(c[k] * idx2); cz[k] = (T)(c[k] * idz2); }
        pp.assign(next(), 0); pc.assign(next(), 0); pn.assign(next(), 0);
        nthreads = (next() >= 65536 && !omp_in_parallel()) ? omp_get_max_threads() : 1;
        return 0;
    }

    // Reference rtm_cpu.cpp:99-123: nearest grid point (lround of the float
    // quotient), clamped to the interior, as an extended-grid index.
    size_t cell(float x, float z) const {
        const int ix0 = (int)std::lround((x - ox) / dx);
        const int iz0 = (int)std::lround((z - oz) / dz);
        const int ix = std::min(std::max(ix0, 0), nx - 1);
        const int iz = std::min(std::max(iz0, 0), nz - 1);
        return e(ix + nb, iz + nb);
    }

    // Reference forward.cpp:29-50.  The outer h-ring is never written.  Every
    // cell is independent, so columns are split over host threads (the result
    // does not depend on the thread count).
    void step() {
#pragma omp parallel for schedule(static) if (nthreads > 1) num_threads(nthreads)
        for (int ix = h; ix < nxe - h; ++ix) {
            for (int iz = h; iz < nze - h; ++iz) {
                const size_t i = e(ix, iz);
                T lap = c0 * pc[i];
                for (int k = 1; k <= h; ++k) {
                    const T ax = pc[i + (size_t)k * nze] + pc[i - (size_t)k * nze];
                    const T az = pc[i + k] + pc[i - k];
                    lap = lap + (cx[k] * ax + cz[k] * az);
                }
                pn[i] = (T)2 * pc[i] - pp[i] + vdt2[i] * lap;
            }
        }
    }

    // Reference forward.cpp:56-63: damp both p^n and p^{n+1} everywhere.
    void damp() {
        const long n = (long)next();
#pragma omp parallel for schedule(static) if (nthreads > 1) num_threads(nthreads)
        for (long i = 0; i < n; ++i) { pc[i] = pc[i] * sponge[i]; pn[i] = pn[i] * sponge[i]; }
    }

    // rotate pp <- pc <- pn (reference forward.cpp:116-118).
    void rotate() { pp.swap(pc); pc.swap(pn); }

    void zero() {
        std::fill(pp.begin(), pp.end(), (T)0);
        std::fill(pc.begin(), pc.end(), (T)0);
        std::fill(pn.begin(), pn.end(), (T)0);
    }

    // Reference forward.cpp:97-125 (step -> inject -> damp -> rotate ->
    // record -> snapshot).  snaps may be null, rec may be null.
    void forward(const oracle_shot& s, T* snaps, T* rec) {
        const size_t src = cell(s.sx, s.sz);
        std::vector<size_t> ridx((size_t)s.nrec);
        for (int ir = 0; ir < s.nrec; ++ir) ridx[ir] = cell(s.rx[ir], s.rz[ir]);
        zero();
        for (int it = 0; it < nt; ++it) {
            step();
            pn[src] = pn[src] + vdt2[src] * wavelet[it];
            damp();
            rotate();
            if (rec)
                for (int ir = 0; ir < s.nrec; ++ir) rec[(size_t)ir * nt + it] = pc[ridx[ir]];
            if (snaps && it % si == 0) {
                T* dst = snaps + (size_t)(it / si) * nint();
                for (int ix = 0; ix < nx; ++ix)
                    for (int iz = 0; iz < nz; ++iz)
                        dst[(size_t)ix * nz + iz] = pc[e(ix + nb, iz + nb)];
            }
        }
    }

    // Reference backward.cpp:20-27 and :40-75 with imaging.cpp:25-40.
    // trace_nt is the stride of the shot's traces (the shot's own nt).  The
    // sums may be kept in a wider type A than the field (test use: FP32
    // propagation and products, FP64 sums).
    template <typename A>
    void backward(const oracle_shot& s, int trace_nt, const T* snaps, A* img, A* ill) {
        std::vector<size_t> ridx((size_t)s.nrec);
        for (int ir = 0; ir < s.nrec; ++ir) ridx[ir] = cell(s.rx[ir], s.rz[ir]);
        zero();
        for (int it = nt - 1; it >= 0; --it) {
            step();
            for (int ir = 0; ir < s.nrec; ++ir) {
                const size_t c = ridx[ir];
                pn[c] = pn[c] + vdt2[c] * (T)s.traces[(size_t)ir * trace_nt + it];
            }
            damp();
            rotate();
            if (it % si == 0) {
                const T* f = snaps + (size_t)(it / si) * nint();
                for (int ix = 0; ix < nx; ++ix)
                    for (int iz = 0; iz < nz; ++iz) {
                        const size_t i = (size_t)ix * nz + iz;
                        const T fv = f[i];
                        const T pi = fv * pc[e(ix + nb, iz + nb)];
                        const T si2 = fv * fv;
                        img[i] = img[i] + (A)pi;
                        ill[i] = ill[i] + (A)si2;
                    }
            }
        }
    }
};

// Reference rtm.cpp:83-103: image/illum zeroed, forward + backward per shot,
// one running image across shots.
template <typename T, typename A = T>
int migrate_impl(const oracle_params* p, const float* vel, int nshots,
                 const oracle_shot* shots, A* image, A* illum) {
    Problem<T> pr;
    const int rc = pr.setup(*p, vel);
    if (rc) return rc;
    std::fill(image, image + pr.nint(), (A)0);
    std::fill(illum, illum + pr.nint(), (A)0);
    std::vector<T> snaps((size_t)pr.nsnap * pr.nint(), (T)0);
    for (int is = 0; is < nshots; ++is) {
        const int trace_nt = shots[is].nt > 0 ? shots[is].nt : p->nt;
        if (trace_nt < p->nt) return -6;
        if (!shots[is].traces) return -5;
        pr.forward(shots[is], snaps.data(), nullptr);
        pr.backward(shots[is], trace_nt, snaps.data(), image, illum);
    }
    return 0;
}

// Reference rtm.cpp:105-111.
template <typename T>
int model_impl(const oracle_params* p, const float* vel, const oracle_shot* s, T* out) {
    Problem<T> pr;
    const int rc = pr.setup(*p, vel);
    if (rc) return rc;
    std::fill(out, out + (size_t)s->nrec * pr.nt, (T)0);
    pr.forward(*s, nullptr, out);
    return 0;
}

}  // namespace

extern "C" {

int oracle_migrate_f32(const oracle_params* p, const float* vel, int nshots,
                       const oracle_shot* shots, float* image, float* illum) {
    return migrate_impl<float>(p, vel, nshots, shots, image, illum);
}
int oracle_migrate_f64(const oracle_params* p, const float* vel, int nshots,
                       const oracle_shot* shots, double* image, double* illum) {
    return migrate_impl<double>(p, vel, nshots, shots, image, illum);
}
int oracle_migrate_f32_sum64(const oracle_params* p, const float* vel, int nshots,
                             const oracle_shot* shots, double* image, double* illum) {
    return migrate_impl<float, double>(p, vel, nshots, shots, image, illum);
}
int oracle_model_shot_f32(const oracle_params* p, const float* vel,
                          const oracle_shot* shot, float* out) {
    return model_impl<float>(p, vel, shot, out);
}
int oracle_model_shot_f64(const oracle_params* p, const float* vel,
                          const oracle_shot* shot, double* out) {
    return model_impl<double>(p, vel, shot, out);
}

int oracle_model_shots_f32(const oracle_params* p, const float* vel, int nshots,
                           const oracle_shot* shots, float* out, int nthreads) {
    int rc_all = 0;
    size_t off = 0;
    std::vector<size_t> offs((size_t)nshots);
    for (int is = 0; is < nshots; ++is) { offs[is] = off; off += (size_t)shots[is].nrec * p->nt; }
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads > 0 ? nthreads : omp_get_max_threads())
    for (int is = 0; is < nshots; ++is) {
        const int rc = model_impl<float>(p, vel, &shots[is], out + offs[is]);
        if (rc) {
#pragma omp critical
            rc_all = rc;
        }
    }
    return rc_all;
}

// Reference seismic_io.cpp:18-35.
void oracle_mute_direct_wave(float sx, float sz, int nrec, const float* rx,
                             const float* rz, int nt, float dt, float* traces,
                             float v_surface, float t_pad, float t_taper) {
    if (v_surface <= 0.0f) return;
    for (int ir = 0; ir < nrec; ++ir) {
        const float ddx = rx[ir] - sx, ddz = rz[ir] - sz;
        const float off = std::sqrt(ddx * ddx + ddz * ddz);
        const float t0 = off / v_surface + t_pad;
        const int i0 = (int)(t0 / dt);
        const int i1 = i0 + std::max(1, (int)(t_taper / dt));
        float* tr = traces + (size_t)ir * nt;
        for (int it = 0; it < nt && it < i1; ++it) {
            if (it <= i0) { tr[it] = 0.0f; continue; }
            const float u = (float)(it - i0) / (float)(i1 - i0);
            tr[it] = tr[it] * (0.5f * (1.0f - std::cos((float)M_PI * u)));
        }
    }
}

float oracle_ricker(float t, float f0) { return ricker_f(t, f0); }

// Reference rtm.cpp:43-62.
float oracle_max_stable_dt(float vmax, float dx, float dz, int order) {
    float c[7];
    const int h = coefficients(order, c);
    if (h < 0) return -1.0f;
    float S = std::fabs(c[0]);
    for (int k = 1; k <= h; ++k) S += 2.0f * std::fabs(c[k]);
    return 2.0f / (vmax * std::sqrt(S * (1.0f / (dx * dx) + 1.0f / (dz * dz))));
}

int oracle_stencil_coefficients(int order, float* out) { return coefficients(order, out); }

}  // extern "C"
