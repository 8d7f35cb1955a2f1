/*
 * mpmw_xpbd.h -- C ABI of the XPBD part of libmpmw.so (spatial hash, contact
 * Jacobi passes, sleeping, MPM contact impulses, swelling).  Conventions as in
 * mpmw.h: device pointers, SoA float[3][n] vec3 fields, int status returns,
 * stream-ordered, no allocation (the hash build takes a caller workspace).
 *
 * Reference citations are to the MPMWarpYDW project (utils/...).
 */
#ifndef MPMW_XPBD_H
#define MPMW_XPBD_H

#include "mpmw.h"

#ifdef __cplusplus
extern "C" {
#endif

/* XPBDState temporaries and per-particle XPBD fields (utils/simStates.py:133-179). */
typedef struct mpmw_xpbd {
    float *x_int, *v_int;        /* [3][n] particle_x/v_integrated */
    float *x_dI, *v_dI;          /* [3][n] particle_x/v_deltaInt (may be NULL) */
    float *delta;                /* [3][n] particle_delta */
    float *v_before;             /* [3][n] particle_v_before_contact (may be NULL) */
    float *cum_dist;             /* [n] particle_cumDist_xpbd */
    float *base_radius, *max_radius; /* [n] particleBaseRadius, particleMaxRadius */
    int32_t *counts;             /* device [2]: numTotalXPBD, numSleepingXPBD (may be NULL) */
} mpmw_xpbd_t;

/* wp.HashGrid(dims) state after build(points, cell_width) (utils/simStates.py:174,
 * utils/simulationRoutines.py:311). */
typedef struct mpmw_hash {
    int32_t dims[3];
    float cell_width;
    int32_t *point_ids;          /* [n] point index at each sorted position */
    int32_t *cell_starts;        /* [dims product] first sorted position of each hash, 0 if empty */
    int32_t *cell_ends;          /* [dims product] one past the last, 0 if empty */
    int32_t *point_cells;        /* [n] hash of each point in input order (may be NULL) */
} mpmw_hash_t;

/* XPBDState scalars + SimState.gravity/dtxpbd (utils/simStates.py:133-179). */
typedef struct mpmw_xpbd_params {
    float gravity[3];
    float dt;                    /* dtxpbd */
    float v_max;                 /* particle_v_max */
    int32_t iterations;          /* xpbd_iterations */
    float relaxation;            /* xpbd_relaxation */
    float coupling;              /* xpbd_mpm_coupling_strength */
    int32_t lock;                /* mpm_contact_transition_lock */
    float dyn_friction;          /* dynamicParticleFriction (k_mu / mu) */
    float static_friction;       /* staticParticleFriction */
    float static_thr;            /* staticVelocityThreshold */
    float cohesion;              /* particle_cohesion (a gap length) */
    float max_radius;            /* XPBDState.max_radius */
    float sleep_thr;             /* sleepThreshold */
    float bmin[3], bmax[3];      /* minBoundsXPBD, maxBoundsXPBD */
    float swelling_ratio, swell_act, swell_max;
    int32_t xpbd_only;
} mpmw_xpbd_params_t;

/* kernel selectors of mpmw_xpbd_kernel */
#define MPMW_XK_INTEGRATE 0    /* xpbdRoutines.py:23-48; flag bit0: read x/v from particles (else x_int/v_int),
                                  flag bit1: also copy non-XPBD particles (the wp.copy before it) */
#define MPMW_XK_RESET_LABELS 1 /* xpbdRoutines.py:3-21 */
#define MPMW_XK_BOUND 2        /* xpbdRoutines.py:49-136; flag: add into delta instead of overwriting it */
#define MPMW_XK_PARTICLE 3     /* xpbdRoutines.py:138-219 (needs a built hash) */
#define MPMW_XK_APPLY 4        /* xpbdRoutines.py:221-257 in place on x_int/v_int; flag: also write x_dI/v_dI */
#define MPMW_XK_SLEEP 5        /* xpbdRoutines.py:312-334; flag: zero counts first */
#define MPMW_XK_IMPULSES 6     /* xpbdRoutines.py:259-310 + the commit x <- x_int, v <- v_int
                                  (simulationRoutines.py:444-470) */
#define MPMW_XK_SWELL 7        /* xpbdRoutines.py:354-375 */

/* Workspace bytes needed by mpmw_hash_build for n points. */
size_t mpmw_hash_workspace_bytes(int64_t n);
/* wp.HashGrid.build (simulationRoutines.py:311): x is [3][n] SoA. */
int mpmw_hash_build(const float *x, int64_t n, const mpmw_hash_t *h, void *workspace, size_t ws_bytes,
                    mpmw_stream_t stream);
/* No counterpart in the reference.  mpmw_hash_build without a caller workspace:
 * for callers that cannot allocate device memory when they build the hash (a
 * host embedding the solver under a fixed device-memory budget, or a loop that
 * must not call cudaMalloc once stepping has started).  Its scratch is a
 * 13 MiB static device array inside the library, so n is limited to
 * MPMW_HASH_NOALLOC_MAX_POINTS; larger n returns MPMW_E_ARG.  The first call on
 * a device (that device current) resolves the array's address; make it before
 * any stream capture.  The address is cached for the life of the process, so
 * do not call this on a device after cudaDeviceReset.  All calls on a device
 * share the array: calls whose GPU work overlaps race on it, so order them on
 * one stream. */
#define MPMW_HASH_NOALLOC_MAX_POINTS 1048576
int mpmw_hash_build_noalloc(const float *x, int64_t n, const mpmw_hash_t *h, mpmw_stream_t stream);
/* One XPBD kernel (MPMW_XK_*). */
int mpmw_xpbd_kernel(int which, const mpmw_particles_t *p, const mpmw_xpbd_t *x, const mpmw_hash_t *h,
                     const mpmw_xpbd_params_t *q, int flag, mpmw_stream_t stream);
/* Bytes of workspace mpmw_xpbd_step uses best for n points on a hash of the
 * given dims: the hash build's scratch, and after the build a count, one bit
 * per hash cell and per-point contact records (mpmw_hash_workspace_bytes(n)
 * is enough; the step then skips the records). */
size_t mpmw_xpbd_step_workspace_bytes(int64_t n, const int32_t *dims);
/* utils/simulationRoutines.py:295-526 xpbdSimulationStep (hash build, integrate,
 * label reset, iterations x (bound, particle contacts, apply), sleep,
 * impulses + commit, swelling).
 * With a workspace of mpmw_xpbd_step_workspace_bytes(n, h->dims) (256-byte
 * aligned) the whole step is ONE persistent kernel: a cooperative launch of
 * at most one full wave of CTAs that runs the hash build, the iterations and
 * the closing passes as phases separated by grid barriers.  Each barrier wait
 * is bounded (1 s); a CTA that gives up sets MPMW_ST_TIMEOUT in *status (may
 * be NULL) and the launch ends early.  With a smaller workspace, or after
 * mpmw_xpbd_set_options(0), one kernel per pass (hash build included).  Both
 * forms give the same bits. */
int mpmw_xpbd_step(const mpmw_particles_t *p, const mpmw_xpbd_t *x, const mpmw_hash_t *h,
                   const mpmw_xpbd_params_t *q, uint32_t *status, void *workspace, size_t ws_bytes,
                   mpmw_stream_t stream);
/* Process-wide form of mpmw_xpbd_step: persistent (1, the default) or one
 * launch per pass (0). */
int mpmw_xpbd_set_options(int persistent);
/* Persistent launches mpmw_xpbd_step has made in this process. */
int64_t mpmw_xpbd_persistent_launches(void);

/* ---- the big step on the device (runMPMYDW.py:633-844) ------------------ */
/* Phase 1 with its XPBD steps and gravity pulse inside one CUDA graph: a while
 * node whose body runs `loop.chunk` fused substeps with the pulse parameters
 * (prm_pulse, q_pulse) while the substep index is below pulse_steps and the
 * plain ones after (the chunk the pulse ends in is split at that substep), an
 * XPBD step after every substep whose index is a positive multiple of
 * xpbd_ratio (runMPMYDW.py:677-682), then the statistics and the driver's
 * check of mpmw_loop_* (residual, damage stall, n_steps, segment budget).  IF
 * nodes pick the branches per chunk, so the launch leaves the graph only when
 * the phase ends or the segment budget runs out.
 * Chunks start at counters = phase (mod chunk); with XPBD steps chunk must
 * divide xpbd_ratio and phase must be 1 mod chunk, so every XPBD substep ends a
 * chunk.  The caller runs the substeps before the first aligned counter.
 * Everything passed is baked into the graph: keep it alive and unchanged. */
typedef struct mpmw_phase_params {
    mpmw_loop_params_t loop;
    int32_t xpbd_ratio;          /* mpmStepsPerXpbdStep; 0: no XPBD steps */
    int32_t pulse_steps;         /* substeps of the gravity pulse from counter 0; 0: none */
    int32_t phase;               /* chunks start at counters = phase (mod loop.chunk) */
} mpmw_phase_params_t;
int mpmw_phase_loop_create(const mpmw_particles_t *p, const mpmw_grid_t *g, const mpmw_params_t *prm,
                           const mpmw_params_t *prm_pulse, const mpmw_xpbd_t *x, const mpmw_hash_t *h,
                           const mpmw_xpbd_params_t *q, const mpmw_xpbd_params_t *q_pulse,
                           const mpmw_phase_params_t *pp, mpmw_loop_state_t *state, uint32_t *status,
                           void *workspace, size_t ws_bytes, void *xpbd_workspace, size_t xpbd_ws_bytes,
                           mpmw_loop_t **out, mpmw_stream_t stream);
/* Phase 2 (runMPMYDW.py:780-844): XPBD-only steps (q->xpbd_only set) until
 * max_steps steps ran (state->counter counts them), the segment budget
 * (state->segment_left) runs out, or the sleeping fraction of XPBD particles
 * (x->counts) reaches sleep_ratio (< 1; state->stopped_early = 1).  Launch with
 * mpmw_loop_launch, destroy with mpmw_loop_destroy. */
int mpmw_xpbd_loop_create(const mpmw_particles_t *p, const mpmw_xpbd_t *x, const mpmw_hash_t *h,
                          const mpmw_xpbd_params_t *q, int max_steps, double sleep_ratio, mpmw_loop_state_t *state,
                          uint32_t *status, void *xpbd_workspace, size_t xpbd_ws_bytes, mpmw_loop_t **out,
                          mpmw_stream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* MPMW_XPBD_H */
