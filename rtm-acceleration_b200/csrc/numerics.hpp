// numerics.hpp -- host-side set-up arithmetic of the RTM scheme.
//
// Everything here runs once per model or per shot on the host, in float, with
// the operation order of the reference (src/rtm/rtm.cpp:14-70 and
// src/rtm/rtm_cpu.cpp:9-123) so that the device tables hold the same bits as
// the reference's tables.  Transcendentals (exp in the Ricker wavelet and the
// Cerjan taper) are evaluated by the host C library here, never on the device.
#pragma once
#include <cstddef>
#include <string>
#include <vector>

#include "internal.hpp"

namespace rtmb {

// order/2 for order in {2,4,...,12}, else -1 (reference rtm.cpp:25-41).
int stencil_half(int order);

// Taylor central second-derivative weights c[0..half] as correctly rounded
// floats, computed from the closed form
//   c_k = 2 (-1)^(k+1) (M!)^2 / (k^2 (M-k)! (M+k)!),  c_0 = -2 sum_k 1/k^2
// in exact integer arithmetic (M = half).  These are the same rationals as the
// reference's table (rtm.cpp:14-23).  Returns false for an unsupported order.
bool stencil_coefficients(int order, float* c);

// |c0| + 2 sum |ck| in float, reference order (rtm.cpp:43-49).
float stencil_abs_sum(int order);

// (1 - 2a) exp(-a), a = pi^2 f0^2 t^2 (rtm.cpp:52-55).
float ricker(float t, float f0);

// CFL limit 2 / (vmax sqrt(S (1/dx^2 + 1/dz^2))) (rtm.cpp:59-62).
float max_stable_dt(float vmax, float dx, float dz, int order);

// vmin / (2.5 f0) / max(dx, dz) (rtm.cpp:66-70).
float points_per_wavelength(float vmin, float f0, float dx, float dz);

// Cerjan weight exp(-(alpha (nb - d))^2) for d = distance to the nearer edge
// < nb, else 1 (rtm_cpu.cpp:50-62).
float cerjan_taper(int i, int n, int nb, float alpha);

// Ricker source samples w[it] = ricker(it*dt - 1.2/f0, f0) (rtm_cpu.cpp:67-70).
std::vector<float> ricker_wavelet(int nt, float dt, float f0);

// Stencil coefficients pre-divided by the spacing (rtm_cpu.cpp:75-79).
struct ScaledCoefficients {
    float c0 = 0;
    float cx[kMaxHalf + 1] = {};
    float cz[kMaxHalf + 1] = {};
};
ScaledCoefficients scaled_coefficients(int order, float dx, float dz);

// Grid of one shot's extended domain and its device pitches.
struct GridDims {
    int nx = 0, nz = 0, nb = 0, half = 0;
    int nxe = 0, nze = 0;
    int ldz = 0;      // field column pitch: nze rounded up to 8 (32-byte columns)
    int zs0 = 0;      // first stored row of snapshots/images: nb rounded down to 4
    int lds = 0;      // stored rows: [zs0, round_up4(nb+nz))
    int ntz = 0;      // 128-row tiles covering nze (from row z0)
    int z0 = 0;       // first row of the 128-row bands; rows above them and below
                      // the last one belong to the zero ring (engine jobs only)
};
GridDims make_grid(int nx, int nz, int nb, int half);

}  // namespace rtmb
