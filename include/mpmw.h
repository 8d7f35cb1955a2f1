/*
 * mpmw.h -- C ABI of libmpmw.so, the B200 (sm_100a) MPM-XPBD substep library.
 *
 * Plain C: raw device pointers, sizes and POD structs; no C++ or torch types
 * cross this boundary, no C++ exception escapes it.  Every entry point returns
 * an int status (MPMW_OK or an MPMW_E_* code) and records a message readable
 * with mpmw_last_error() (thread-local).  Entry points are stream-ordered: they
 * enqueue work on `stream` and never synchronize the host, never allocate
 * device memory, and write device-side faults (out-of-grid stencil, NaN) into
 * the caller's device status word (`status`, may be NULL).
 *
 * Data layout (all float32 unless stated; "SoA" = component-major):
 *   vec3 field  : float[3][n]      component c of particle p at ptr[c*n + p]
 *   mat33 field : float[9][n]      entry (r,c) at ptr[(3r+c)*n + p]
 *   stress      : float[6][n]      xx, yy, zz, xy, xz, yz (symmetric)
 *   cov         : float[n][6]      reference layout (utils/mpmRoutines.py:779-802)
 *   grid mv     : float[G][4]      (m, m*vx, m*vy, m*vz) P2G accumulators
 *   grid v      : float[G][4]      (vx, vy, vz, 0) grid velocity
 *   node (ix,iy,iz) -> (ix*ny + iy)*nz + iz   (C order, z fastest)
 *
 * Reference citations are to the MPMWarpYDW project (utils/...).
 */
#ifndef MPMW_H
#define MPMW_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* return codes */
#define MPMW_OK 0
#define MPMW_E_ARG 1        /* invalid argument (null pointer, size, enum) */
#define MPMW_E_LAUNCH 2     /* kernel launch failed */
#define MPMW_E_DEVICE 3     /* CUDA runtime error */
#define MPMW_E_WORKSPACE 4  /* workspace too small */

/* device status word bits (OR-ed by kernels into *status) */
#define MPMW_ST_OOB 1u      /* a stencil node fell outside the grid; access skipped */
#define MPMW_ST_NAN 2u      /* a non-finite particle position was produced */
#define MPMW_ST_TIMEOUT 4u  /* a bounded wait gave up */

/* boundary condition codes (utils/simulationRoutines.py:124-228) */
#define MPMW_BC_NONE -1
#define MPMW_BC_FRICTION 0
#define MPMW_BC_FRICTION_GRADUAL 1
#define MPMW_BC_RESTITUTION 2
#define MPMW_BC_ABSORBING 3
#define MPMW_BC_PLANE_STRAIN_Y 4
#define MPMW_BC_PLANE_STRAIN_Y_GLOBAL 5

typedef void *mpmw_stream_t; /* a cudaStream_t; NULL = legacy default stream */

/* Per-particle arrays (utils/simStates.py:10-179 SimState/MPMState/XPBDState). */
typedef struct mpmw_particles {
    int64_t n;
    float *x, *v;                /* [3][n] particle_x, particle_v */
    float *C, *F, *F_trial;      /* [9][n] particle_C, particle_F, particle_F_trial */
    float *stress;               /* [6][n] particle_stress (symmetric) */
    float *cov;                  /* [n][6] particle_cov, may be NULL if update_cov == 0 */
    float *vol, *mass, *density, *radius;
    float *mu, *lam, *ys, *alpha, *hardening, *softening, *strain_criteria;
    float *eta_shear, *eta_bulk;
    float *acc_strain, *damage;  /* particle_accumulated_strain, particle_damage */
    int32_t *active, *material;  /* activeLabel, materialLabel */
    float *x_pc, *v_pc;          /* [3][n] particle_x/v_initial_xpbd (phase-change records) */
} mpmw_particles_t;

/* One background grid. */
typedef struct mpmw_grid {
    int32_t dims[3];
    float *mv;                   /* [G][4] grid_m + grid_v_in */
    float *v;                    /* [G][4] grid_v_out */
    float *cell_div, *cell_vol;  /* [G] cell_div_v_weighted, cell_vol_sum (VLC only) */
} mpmw_grid_t;

/* Scalars of one MPM scene (SimState/MPMState scalars + getArgs flags). */
typedef struct mpmw_params {
    float min_bounds[3];
    float dx, inv_dx, dt;
    float gravity[3];            /* already scaled by any gravity pulse */
    float rpic_damping;
    float grid_v_damping_scale;  /* applied only when < 1 */
    float bound_friction, bound_restitution;
    int32_t boundary_condition;  /* MPMW_BC_* */
    int32_t boundary_padding;
    float eff;                   /* phase-change energy efficiency */
    int32_t update_cov;
    int32_t vlc;                 /* volumetric_locking_correction */
    int32_t constitutive_model;  /* accepted and ignored, as in the reference */
    int32_t stress_mode;         /* MPMW_STRESS_* */
} mpmw_params_t;

/* stress_mode: how the return map is evaluated (same model either way).
 *   MPMW_STRESS_AUTO (0): when |F F^T - I|_F <= 0.02 the return map runs in
 *     tensor form on the spatial log strain eps = 1/2 ln(I + X),
 *     X = G + G^T + G G^T, G = F - I (series): invariants for the yield test,
 *     radial return on dev(eps), F_e = e^vc exp(-f dev eps) F, Kirchhoff stress
 *     2 mu eps + lam tr(eps) I.  This is the reference's principal-space algebra
 *     without an SVD, and it avoids FP32 rounding of ln(s) for s near 1.  Larger
 *     deformations take the SVD path.
 *   MPMW_STRESS_SVD (1): every particle takes the SVD path (svd3 of F_trial,
 *     principal log strains, radial return, second svd3 for the Kirchhoff
 *     stress), operation for operation as the CPU oracle. */
#define MPMW_STRESS_AUTO 0
#define MPMW_STRESS_SVD 1

/* ---- library ------------------------------------------------------------ */
const char *mpmw_last_error(void);
int mpmw_version(void);

/* ---- set-up kernels ------------------------------------------------------ */
/* utils/mpmRoutines.py:206-226 compute_mu_lam_bulk_from_E_nu */
int mpmw_mu_lam_bulk(int64_t n, const float *E, const float *nu, float *mu, float *lam, float *bulk,
                     mpmw_stream_t stream);
/* utils/mpmRoutines.py:51-124 initialize_geostatic_F (planestrain != 0:
 * :127-203 initialize_geostatic_F_planestrain); F is [9][n] SoA */
int mpmw_geostatic_F(int64_t n, const float *x, float *F, const float *mu, const float *lam,
                     const float *density, float gravity, float z_top, float K0, int planestrain,
                     mpmw_stream_t stream);

/* ---- MPM substep kernels ------------------------------------------------- */
/* utils/mpmRoutines.py:229-312 compute_stress_from_F_trial (+ :314-453 return map,
 * :456-471 Kirchhoff stress) */
int mpmw_stress(const mpmw_particles_t *p, const mpmw_params_t *prm, uint32_t *status, mpmw_stream_t stream);
/* utils/mpmRoutines.py:485-569 p2g_apic_with_stress (accumulates into grid->mv;
 * the caller zeroes it first, utils/simulationRoutines.py:11-13) */
int mpmw_p2g(const mpmw_particles_t *p, const mpmw_grid_t *g, const mpmw_params_t *prm, uint32_t *status,
             mpmw_stream_t stream);
/* utils/mpmRoutines.py:690-711 grid_normalization_and_gravity + add_damping_via_grid,
 * fused with the boundary kernel selected at utils/simulationRoutines.py:124-228
 * (mpmRoutines.py:914-1362).  Writes every node of grid->v. */
int mpmw_grid_update(const mpmw_grid_t *g, const mpmw_params_t *prm, mpmw_stream_t stream);
/* One reference grid kernel on its own, with its exact write set:
 *   op 0  utils/mpmRoutines.py:690-704 grid_normalization_and_gravity (nodes with
 *         m <= 1e-15 are left untouched)
 *   op 1  utils/mpmRoutines.py:706-711 add_damping_via_grid (scale by
 *         prm->grid_v_damping_scale, unconditionally)
 *   op 2  the boundary kernel prm->boundary_condition (mpmRoutines.py:914-1362) */
int mpmw_grid_op(const mpmw_grid_t *g, const mpmw_params_t *prm, int op, mpmw_stream_t stream);
/* utils/mpmRoutines.py:715-802 g2p (+ update_cov) */
int mpmw_g2p(const mpmw_particles_t *p, const mpmw_grid_t *g, const mpmw_params_t *prm, uint32_t *status,
             mpmw_stream_t stream);
/* g2p followed, per particle and in registers, by the next substep's
 * compute_stress_from_F_trial (including Kelvin-Voigt from the new C).  Writes
 * F (returned) and stress instead of F_trial.  Equivalent to mpmw_g2p followed
 * by mpmw_stress when nothing runs between them (no VLC, no XPBD). */
int mpmw_g2p_stress(const mpmw_particles_t *p, const mpmw_grid_t *g, const mpmw_params_t *prm,
                    uint32_t *status, void *workspace, size_t ws_bytes, mpmw_stream_t stream);
/* Bytes of device workspace mpmw_g2p_stress / mpmw_run_substeps need for n
 * particles (a worklist of the particles whose return map takes the SVD path). */
size_t mpmw_workspace_bytes(int64_t n);
/* utils/mpmRoutines.py:229-312 compute_stress_from_F_trial followed by
 * :485-569 p2g_apic_with_stress (the launches at utils/simulationRoutines.py:15-69)
 * in one pass: F and the stress are written as mpmw_stress writes them and the
 * scatter accumulates into grid->mv as mpmw_p2g does (the caller zeroes it).
 * Needs mpmw_workspace_bytes(n) of workspace for the SVD-path worklist. */
int mpmw_stress_p2g(const mpmw_particles_t *p, const mpmw_grid_t *g, const mpmw_params_t *prm, uint32_t *status,
                    void *workspace, size_t ws_bytes, mpmw_stream_t stream);
/* The middle of a fused run (utils/simulationRoutines.py:6-293 applied twice):
 * substep k's g2p (mpmRoutines.py:715-802), then substep k+1's
 * compute_stress_from_F_trial (:229-312) and p2g_apic_with_stress (:485-569),
 * per particle in registers.  grid->v holds substep k's grid velocity and
 * grid->mv must be zero on entry (it receives substep k+1's P2G).  Writes x and
 * F; the stress only when store_stress != 0; v, C and F_trial only for
 * particles that leave the MPM path or need the SVD return map.  A run of such
 * calls ends with mpmw_g2p, which writes x, v, C and F_trial. */
int mpmw_g2p2g(const mpmw_particles_t *p, const mpmw_grid_t *g, const mpmw_params_t *prm, int store_stress,
               uint32_t *status, void *workspace, size_t ws_bytes, mpmw_stream_t stream);
/* utils/mpmRoutines.py:817-911 accumulate_cell_divergence + apply_volumetric_locking_correction
 * (zeroes grid->cell_div / cell_vol itself, utils/simulationRoutines.py:255-293) */
int mpmw_vlc(const mpmw_particles_t *p, const mpmw_grid_t *g, const mpmw_params_t *prm, uint32_t *status,
             mpmw_stream_t stream);
/* One phase of the correction on its own: phase 0 = accumulate_cell_divergence
 * (mpmRoutines.py:817-856, adds into grid->cell_div / cell_vol, no zeroing),
 * phase 1 = apply_volumetric_locking_correction (mpmRoutines.py:859-911).
 * Only grid->dims, cell_div and cell_vol are used. */
int mpmw_vlc_phase(const mpmw_particles_t *p, const mpmw_grid_t *g, const mpmw_params_t *prm, int phase,
                   uint32_t *status, mpmw_stream_t stream);
/* utils/simulationRoutines.py:6-293 mpmSimulationStep: zero grid, stress, P2G,
 * grid update, G2P, optional VLC -- one reference substep */
int mpmw_substep(const mpmw_particles_t *p, const mpmw_grid_t *g, const mpmw_params_t *prm, uint32_t *status,
                 mpmw_stream_t stream);
/* nsteps consecutive mpmSimulationStep calls with no XPBD between them
 * (runMPMYDW.py:666-682 for steps where counter % mpmStepsPerXpbdStep != 0).
 * Same result as nsteps x mpmw_substep; when VLC is off and a workspace of
 * mpmw_workspace_bytes(n) is given, the return map of step k+1 runs fused into
 * the G2P of step k. */
int mpmw_run_substeps(const mpmw_particles_t *p, const mpmw_grid_t *g, const mpmw_params_t *prm, int nsteps,
                      uint32_t *status, void *workspace, size_t ws_bytes, mpmw_stream_t stream);

/* ---- batched independent scenes (parameter sweeps) ----------------------- */
#define MPMW_BATCH_MAX_SCENES 192  /* scenes per batch (their grid tensor maps travel as a kernel parameter) */
/* Many independent scenes stepped together, each kernel one launch over all of
 * them (runMPMYDW.py:666-682 steps of independent scenes; the batching has no
 * reference counterpart).  The scenes' particles are concatenated in the SoA
 * arrays of *p: scene s owns particles [offsets[s], offsets[s+1]), every offset
 * a multiple of 256 (a scene is padded with inactive particles, active = 0),
 * offsets[0] = 0 and offsets[nscenes] = p->n.  grids[s] and prms[s] are scene
 * s's grid and parameters; VLC must be off.
 *
 * Bytes of workspace for such a batch: the SVD worklist (n ints), a worklist
 * count per scene and the scene table. */
size_t mpmw_batch_workspace_bytes(const mpmw_grid_t *grids, int nscenes, int64_t n);
/* Checks the batch (1 <= nscenes <= MPMW_BATCH_MAX_SCENES) and writes its scene
 * table (each scene's grid and parameters; each CTA's scene) into the
 * workspace; the library keeps the scenes' grid tensor maps for the run.
 * Synchronizes `stream`; run it again after changing a grid, a parameter or
 * the offsets. */
int mpmw_batch_prepare(const mpmw_particles_t *p, const mpmw_grid_t *grids, const mpmw_params_t *prms,
                       const int64_t *offsets, int nscenes, void *workspace, size_t ws_bytes, mpmw_stream_t stream);
/* nsteps substeps of every scene of the batch prepared in this workspace: per
 * scene the same result as mpmw_run_substeps on that scene alone.  No host
 * synchronization (capturable in a CUDA graph). */
int mpmw_batch_run_substeps(const mpmw_particles_t *p, int nsteps, uint32_t *status, void *workspace,
                            size_t ws_bytes, mpmw_stream_t stream);
/* The same for the scenes [first_scene, last_scene) of the prepared batch.
 * Disjoint ranges use disjoint particles, grids and worklists, so they may run
 * concurrently on different streams (how many ranges suits a batch best is
 * measured by sweep.ConcatBatch.tune). */
int mpmw_batch_run_range(const mpmw_particles_t *p, int first_scene, int last_scene, int nsteps, uint32_t *status,
                         void *workspace, size_t ws_bytes, mpmw_stream_t stream);
/* The same nsteps substeps of every scene with the fused substeps of all
 * scenes in ONE persistent kernel: a cooperative launch of at most one full
 * wave that runs, per substep, the grid update of every scene's grid, the
 * fused G2P -> return map -> P2G of every scene's particles (particle tiles
 * handed out as CTAs free up) and the SVD worklist, separated by grid
 * barriers.  Before it, the prologue (grids cleared, the first return map and
 * P2G); after it, the last grid update and G2P.  Same results as
 * mpmw_batch_run_substeps.  Each barrier wait is bounded (1 s): a CTA that
 * gives up sets MPMW_ST_TIMEOUT and the launch ends early.  Not to be run
 * concurrently with another persistent launch. */
int mpmw_batch_run_persistent(const mpmw_particles_t *p, int nsteps, uint32_t *status, void *workspace,
                              size_t ws_bytes, mpmw_stream_t stream);
/* Persistent batch launches made in this process. */
int64_t mpmw_batch_persistent_launches(void);

/* ---- particle order ------------------------------------------------------ */
/* No counterpart in the reference (its kernels do not depend on particle
 * order, utils/mpmRoutines.py:485-569).  perm[n] receives the stable order of
 * the particles by block key: each particle's stencil base cell
 * int((x - min_bounds) inv_dx - 0.5) per axis (utils/mpmRoutines.py:514-517),
 * clamped to the grid `dims`, grouped in blocks of block^3 cells -- key =
 * (block index, C order) * block^3 + (cell within the block, C order) -- by
 * the library's stable LSD radix sort.  Position i of the sorted order holds
 * particle perm[i].  x is [3][n] SoA; prm supplies min_bounds and inv_dx.
 * Gathering every particle field through perm keeps the particles a CTA of
 * the scatter and gather kernels holds within a few cells.  Needs
 * mpmw_block_sort_workspace_bytes(n) of workspace; the number of keys must
 * stay below 2^31. */
size_t mpmw_block_sort_workspace_bytes(int64_t n);
int mpmw_block_sort(const float *x, int64_t n, const mpmw_params_t *prm, const int32_t *dims, int block,
                    int32_t *perm, void *workspace, size_t ws_bytes, mpmw_stream_t stream);

/* Launch options of the batch prepared in this workspace (no counterpart in
 * the reference; what sweep.ConcatBatch.tune searches): gather_tile != 0 lets
 * a CTA load its grid tile by TMA (else the gather reads the grid through L1),
 * read_ahead != 0 lets it read its particle fields ahead by bulk copies (else
 * plain loads).  Either is used only where mpmw_batch_prepare found it usable;
 * the results are the same either way.  Host-side only: no device work. */
int mpmw_batch_set_options(const void *workspace, int gather_tile, int read_ahead);

/* utils/mpmRoutines.py:1446-1475 deactivate_and_teleport_xpbd_below_datum */
int mpmw_teleport(const mpmw_particles_t *p, float z_datum, float teleport_distance, mpmw_stream_t stream);
/* utils/mpmRoutines.py:3-21 creep_by_damage_with_baseline */
int mpmw_creep(const mpmw_particles_t *p, const float *ys_base, float dt, float base_creep, float damage_creep,
               float damage_exponent, mpmw_stream_t stream);

/* ---- per-step statistics (utils/simulationRoutines.py:538-675) ----------- */
/* out (device, 7 doubles, 8-byte aligned, overwritten): sum |v|/radius over active
 * (velocityConvergence), active count (countActiveParticles), sum damage over active
 * (compute_mean_gpu numerator), active MPM, active XPBD, inactive MPM, inactive XPBD
 * (countParticlesByType).  The sums are accumulated in FP32 (compensated per thread,
 * pairwise per block, one FP32 atomic per block), the counts in integers; only the
 * final conversion writes doubles.  Two launches. */
int mpmw_stats(const mpmw_particles_t *p, double *out, mpmw_stream_t stream);

/* ---- phase-1 loop on the device (runMPMYDW.py:656-727) ------------------ */
/* The reference driver runs substeps while counter < nSteps and (counter <
 * minSteps or residual > residualThreshold), ending early when the mean
 * damage stalls, and reads the residual back to the host every substep.  A
 * loop object runs that test on the device: one CUDA graph whose while-node
 * body is `chunk` fused substeps (mpmw_run_substeps), the statistics
 * (mpmw_stats) and a decision kernel, so a launch runs chunk after chunk with
 * no host round trip until the phase ends or `segment_left` runs out.  The
 * decision is the driver's check made every `chunk` substeps, in double
 * precision: counter += chunk; residual = sum|v|/r / active; the damage
 * stall counter grows by chunk when mean damage rose by less than
 * stall_threshold * chunk and counter > min_steps, else resets; the phase
 * ends early when stall >= stall_steps and counter > min_steps. */
typedef struct mpmw_loop_state { /* device memory, 8-byte aligned */
    int counter;       /* substeps run in the phase */
    int stall;         /* substeps of stalled damage */
    int stopped_early; /* 1 once the damage stall ended the phase */
    int segment_left;  /* substeps this launch may still run (set by the caller, multiple of chunk) */
    double residual;   /* sum |v|/r / active at the last check (1e10 before any) */
    double prev_damage;/* mean damage over active at the last check */
    double stats[7];   /* mpmw_stats of the last check */
} mpmw_loop_state_t;
typedef struct mpmw_loop_params {
    int chunk, n_steps, min_steps, stall_steps;
    double residual_threshold, stall_threshold;
} mpmw_loop_params_t;
typedef struct mpmw_loop mpmw_loop_t;
/* Builds the graph on `stream` (captured, nothing runs).  The structs, the
 * workspace (mpmw_workspace_bytes(n)) and `state` are baked in: keep them alive
 * and unchanged while the loop exists. */
int mpmw_loop_create(const mpmw_particles_t *p, const mpmw_grid_t *g, const mpmw_params_t *prm,
                     const mpmw_loop_params_t *lp, mpmw_loop_state_t *state, uint32_t *status, void *workspace,
                     size_t ws_bytes, mpmw_loop_t **out, mpmw_stream_t stream);
/* Runs chunks while the phase continues and state->segment_left >= chunk (at
 * least one chunk: launch only when that holds). */
int mpmw_loop_launch(mpmw_loop_t *loop, mpmw_stream_t stream);
void mpmw_loop_destroy(mpmw_loop_t *loop);

#ifdef __cplusplus
}
#endif
#endif /* MPMW_H */
