/*
 * rtm_oracle.h -- C ABI of the CPU oracle (TEST INFRASTRUCTURE ONLY).
 *
 * The oracle is a plain CPU restatement of the reference's 2D acoustic RTM
 * (Marouane-Djabri/RTM-Acceleration, CPUReferenceRTM).  It exists to check the
 * CUDA engine; it is never linked into, loaded by or called from the product
 * library.  Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
 * leg may use it.
 *
 * Two instances of the same template:
 *   *_f32 : float arithmetic, no FMA contraction -> bit-identical to the
 *           reference CPU engine built with its own -O2 flags (pinned by
 *           tests/test_oracle_golden.py against images/traces produced by the
 *           reference binaries and against the reference's recorded SHA-256 of
 *           its Marmousi shot file).
 *   *_f64 : the FP64 oracle: all set-up tables (v^2 dt^2, sponge, Ricker,
 *           FD coefficients) are computed in float exactly as the reference
 *           does, then widened; propagation, injection and imaging run in
 *           double.  "The same scheme in higher precision."
 */
#ifndef RTM_ORACLE_H
#define RTM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int   nx, nz;          /* interior grid                                   */
    float dx, dz, ox, oz;  /* spacing and origin, metres                      */
    int   nb;              /* sponge width (cells)                            */
    int   order;           /* FD order 2..12                                  */
    float sponge_alpha;    /* Cerjan coefficient                              */
    int   store_interval;  /* snapshot cadence                                */
    float f0;              /* Ricker peak frequency                           */
    int   nt;              /* time samples                                    */
    float dt;              /* seconds                                         */
} oracle_params;

typedef struct {
    float        sx, sz;   /* source position, metres                         */
    int          nrec;
    int          nt;       /* samples per trace = stride of traces; 0 means
                              oracle_params.nt.  May exceed params.nt (the
                              reference's --nt truncation, src/main.cpp:162) */
    const float* rx;       /* nrec receiver x, metres                         */
    const float* rz;       /* nrec receiver z, metres                         */
    const float* traces;   /* nrec*nt trace-major (traces[ir*nt+it]); may be
                              NULL for modelling                              */
} oracle_shot;

/* Full migration over all shots (reference RTMEngine::migrate), image and
 * illumination are nx*nz, zfast, overwritten.  Returns 0 on success, <0 on a
 * validation error (same checks as the reference's setup). */
int oracle_migrate_f32(const oracle_params* p, const float* vel, int nshots,
                       const oracle_shot* shots, float* image, float* illum);
int oracle_migrate_f64(const oracle_params* p, const float* vel, int nshots,
                       const oracle_shot* shots, double* image, double* illum);
/* The same with FP32 propagation and FP32 products, exactly as the reference,
 * but the image and illumination summed in FP64: the reference point for the
 * engines' compensated FP32 sums (test infrastructure only). */
int oracle_migrate_f32_sum64(const oracle_params* p, const float* vel, int nshots,
                             const oracle_shot* shots, double* image, double* illum);

/* Forward modelling of one shot (reference RTMEngine::model_shot): writes
 * nrec*nt trace-major samples. */
int oracle_model_shot_f32(const oracle_params* p, const float* vel,
                          const oracle_shot* shot, float* traces_out);
int oracle_model_shot_f64(const oracle_params* p, const float* vel,
                          const oracle_shot* shot, double* traces_out);

/* Many independent shots in parallel over host threads (nthreads<=0: all). */
int oracle_model_shots_f32(const oracle_params* p, const float* vel, int nshots,
                           const oracle_shot* shots, float* traces_out,
                           int nthreads);

/* Direct-wave mute (reference mute_direct_wave), in place on nrec*nt traces. */
void oracle_mute_direct_wave(float sx, float sz, int nrec, const float* rx,
                             const float* rz, int nt, float dt, float* traces,
                             float v_surface, float t_pad, float t_taper);

/* Shared numerics, for checking the product's host set-up code. */
float oracle_ricker(float t, float f0);
float oracle_max_stable_dt(float vmax, float dx, float dz, int order);
int   oracle_stencil_coefficients(int order, float* out /* half+1 */);

#ifdef __cplusplus
}
#endif
#endif
