/*
 * empm_b200.h — C ABI of the B200 (sm_100a) MLS-MPM substep library.
 *
 * This library replaces the Warp kernels and the per-substep launch sequence of
 * EMPM's differentiable MPM simulator (phys_sim/diff_simulator/warp_mpm/).
 * Every function returns an int status (EMPM_OK = 0, negative = error) and
 * takes plain pointers and sizes; device pointers are borrowed (the caller,
 * normally PyTorch, owns them) and the CUDA stream is passed explicitly.
 * A context owns only its own scratch (grid buffers, step tables, status word).
 *
 * Particle layout in HBM ("f4" and "f9" planes, structure of arrays):
 *   x   : float[4*N]  per particle (x, y, z, mass)          -- one float4
 *   v   : float[4*N]  per particle (vx, vy, vz, 0)          -- one float4
 *   C,F : float[9*N]  3x3 row-major matrix split in three planes:
 *         plane A float4[N] = (m00, m01, m02, m10)
 *         plane B float4[N] = (m11, m12, m20, m21)
 *         plane C float [N] = (m22)
 *         plane A starts at the pointer, B at +16*N bytes, C at +32*N bytes.
 * Grid layout: float4 per node, 4x4x4-node blocks (see empm_ctx_grid).
 *
 * Reference interfaces replaced (paths relative to the EMPM repository):
 *   empm_substep        <- MPMWARPDiff.p2g2p_differentiable
 *                          phys_sim/diff_simulator/warp_mpm/mpm_solver_diff.py:165-291
 *                          (kernels zero_grid, compute_stress_from_F_trial,
 *                          p2g_apic_with_stress, grid_normalization_and_gravity,
 *                          add_damping_via_grid, collider closures, g2p_differentiable
 *                          in mpm_utils.py:286-665,722-734 and
 *                          mpm_solver_diff.py:473-528,612-672,756-801,835-866,878-935,1275-1286)
 *   empm_substep_inplace <- MPMWARPDiff.p2g2p (mpm_solver_diff.py:293-429, in-place g2p and
 *                          clip_particle_x, mpm_utils.py:441-499,582-599)
 *   empm_rollout        <- the substep loop of WarpMPMWrapper.advance_to
 *                          warp_mpm_wrapper.py:278-306 and interface.py:137-145
 *   empm_prepare        <- compute_mu_lam_from_E_nu (mpm_utils.py:277-283) and the
 *                          mass = density * vol launch (mpm_data_structure.py:719-726)
 *   empm_pack_particles / empm_unpack_particles
 *                       <- MPMStateStruct.from_torch / continue_from_torch and
 *                          wp.to_torch of particle arrays (mpm_data_structure.py:119-172,257-292)
 *   empm_adjoint_segment <- the Warp tape replay of the substep kernels' adjoints
 *                          (MyTape / tape.backward, warp_utils.py:93-142;
 *                          interface.py:167-251,391-472,579-774,899-986)
 *   empm_segment_*      <- the tape's record of the forward launches kept for the
 *                          reverse pass (MyTape, warp_utils.py:93-127; interface.py:135-145)
 *   empm_prepare_adjoint <- the adjoints of compute_mu_lam_from_E_nu and of the mass
 *                          product on the same tape (mpm_utils.py:277-283,
 *                          mpm_data_structure.py:719-726)
 */
#ifndef EMPM_B200_H
#define EMPM_B200_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EMPM_OK                 0
#define EMPM_ERR_INVALID       -1  /* bad argument (null pointer, size out of range) */
#define EMPM_ERR_CUDA          -2  /* a CUDA runtime call failed; see empm_last_error */
#define EMPM_ERR_OOM           -3  /* device allocation failed */
#define EMPM_ERR_UNSUPPORTED   -4  /* material or option not supported */
#define EMPM_ERR_TIMEOUT       -5  /* a bounded device-side wait gave up */
#define EMPM_ERR_NUMERIC       -6  /* device status word reported NaN/Inf or CFL breach */

#define EMPM_MAX_COLLIDERS  16
#define EMPM_MAX_MODIFIERS  8

/* Device status word bits (empm_read_status). */
#define EMPM_STATUS_NAN          1u   /* non-finite x, v or F written */
#define EMPM_STATUS_CFL          2u   /* |v| * dt > dx for some particle */
#define EMPM_STATUS_OUT_OF_BAND  4u   /* particle stencil outside the grid (clamped) */

/* Material ids, identical to MPMWARPDiff.set_parameters_dict (mpm_solver_diff.py:39-55). */
#define EMPM_MAT_JELLY        0
#define EMPM_MAT_METAL        1
#define EMPM_MAT_SAND         2
#define EMPM_MAT_FOAM         3
#define EMPM_MAT_SNOW         4
#define EMPM_MAT_PLASTICINE   5
#define EMPM_MAT_NEOHOOKEAN   6

/* Scalar model parameters: the scalar fields of MPMModelStruct
 * (mpm_data_structure.py:391-422; defaults in init_other_params :456-484). */
typedef struct {
    int   n_grid;                 /* cubic grid resolution G */
    float grid_lim;               /* domain extent (dx = grid_lim / G) */
    int   material;               /* EMPM_MAT_* */
    float gravity[3];             /* gravitational_accelaration */
    float rpic_damping;           /* 0 = APIC, < -0.001 = PIC */
    float grid_v_damping_scale;   /* < 1 enables add_damping_via_grid */
    float softening;
    float hardening;
    float xi;
    float plastic_viscosity;
    float alpha;                  /* Drucker-Prager alpha from friction_angle */
} EmpmModelParams;

/* Collider kinds: one per factory of MPMWARPDiff. */
#define EMPM_COLL_SURFACE          1  /* add_surface_collider        mpm_solver_diff.py:437-531 */
#define EMPM_COLL_GEOMETRY         2  /* add_geometry_collider       :533-683 */
#define EMPM_COLL_GRID_VELOCITY    3  /* set_grid_velocity_on_geometry :685-804 */
#define EMPM_COLL_CUBOID_VELOCITY  4  /* set_velocity_on_cuboid      :814-869 */
#define EMPM_COLL_BOUNDING_BOX     5  /* add_bounding_box            :871-938 */
#define EMPM_COLL_GRID_MASK        6  /* enforce_grid_velocity_by_mask :1264-1289 */

/* Shapes of the geometry colliders (geo_type in the reference). */
#define EMPM_SHAPE_CUBE       1
#define EMPM_SHAPE_SPHERE     2
#define EMPM_SHAPE_CYLINDER   3
#define EMPM_SHAPE_HALFSPACE  4

/* Per-substep gate decided on the host from the collider's time window
 * (the `time >= start_time and time < end_time` tests of the closures). */
#define EMPM_GATE_OFF        0    /* collider does nothing this substep */
#define EMPM_GATE_APPLY      1    /* apply the collider's shape rule */
#define EMPM_GATE_ZERO_ALL   2    /* reset branch: zero every grid node */

typedef struct {
    int   kind;            /* EMPM_COLL_* */
    int   gate;            /* EMPM_GATE_* for this substep */
    int   shape;           /* EMPM_SHAPE_* (geometry kinds) */
    int   surface_type;    /* 0 sticky, 1 slip, 11 cut, 2 other */
    float point[3];
    float normal[3];       /* unit normal / cylinder axis */
    float size[3];         /* half extents (cube, cuboid) */
    float velocity[3];
    float rot_axis[3];
    float angular_velocity;
    float radius;
    float half_height;
    float friction;
    const int32_t* mask;   /* device [G^3] for EMPM_COLL_GRID_MASK, else NULL */
} EmpmCollider;

/* Particle velocity modifiers applied before P2G (pre_p2g_operations and
 * particle_velocity_modifiers of MPMWARPDiff). */
#define EMPM_MOD_IMPULSE          1  /* add_impulse_on_particles:           v += force/mass*dt (mask==1) :943-991 */
#define EMPM_MOD_IMPULSE_MASK     2  /* add_impulse_on_particles_with_mask: v += force*dt     (mask>=1) :1353-1410 */
#define EMPM_MOD_SET_VELOCITY     3  /* enforce_particle_velocity_translation/_by_mask: v = velocity (mask==1) :993-1036,1173-1212 */
#define EMPM_MOD_ROTATION         4  /* enforce_particle_velocity_rotation  :1041-1142 */
#define EMPM_MOD_MOVER            5  /* set_particle_mover: v += velocity + w * axis x (x - center) :1291-1348 */
#define EMPM_MOD_SET_VELOCITY_LAYERED 6  /* release_particles_sequentially :1146-1171: v = velocity where
                                           mask >= (int)scale[0]; mask counts the nested release boxes that
                                           hold the particle, scale[0] = 1 + the outermost box still held */

typedef struct {
    int   kind;            /* EMPM_MOD_* */
    int   gate;            /* EMPM_GATE_OFF or EMPM_GATE_APPLY for this substep */
    float vec[3];          /* force or velocity */
    float point[3];        /* rotation: cylinder point; mover: rotation center */
    float normal[3];       /* rotation: cylinder axis; mover: rotation axis */
    float axis1[3];        /* rotation: horizontal_axis_1 */
    float axis2[3];        /* rotation: horizontal_axis_2 */
    float scale[2];        /* rotation: rotation_scale, translation_scale; mover: angular velocity in [0] */
    const int32_t* mask;   /* device [N] indexed by the caller's particle order */
} EmpmModifier;

/* One substep's host-side schedule: the solver time (float32 as the kernels
 * see it), dt, and the colliders / modifiers with their gates resolved. */
typedef struct {
    float time;
    float dt;
    int   n_colliders;
    int   n_modifiers;
    int   hold;            /* 1: this instance does not advance in this substep; its particles
                              are copied unchanged (a batch member that has finished while the
                              others continue). Not supported by empm_adjoint_segment. */
    int   reserved;        /* 0 */
    EmpmCollider colliders[EMPM_MAX_COLLIDERS];
    EmpmModifier modifiers[EMPM_MAX_MODIFIERS];
} EmpmStep;

/* Particle state buffers (device pointers, layout in the file header). */
typedef struct {
    float* x;       /* float4 plane (x, y, z, mass) */
    float* v;       /* float4 plane (vx, vy, vz, 0) */
    float* C;       /* f9 planes: APIC affine matrix */
    float* F;       /* f9 planes: trial deformation gradient (particle_F_trial) */
} EmpmParticles;

/* Per-particle material arrays (device pointers, [N] each). */
typedef struct {
    const float*   vol;          /* particle_vol */
    float*         mu;           /* mutated by plasticine (damage) */
    float*         lam;          /* mutated by plasticine (damage) */
    float*         yield_stress; /* mutated by the von Mises return maps */
    const int32_t* selection;    /* particle_selection (0 = simulated) or NULL */
    float*         F_elastic;    /* f9 planes [N]: receives particle_F (post-return-map F) */
} EmpmMaterial;

typedef struct EmpmCtx EmpmCtx;

int  empm_version(void);

/* Create a context for one simulation instance of n_particles on a G^3 grid
 * (a batch of one, see empm_batch_create). Allocates the two grid buffers
 * (2 * 16 * 64 * ceil(G/4)^3 bytes), room for max_steps step tables and the
 * status word on the current device. */
int  empm_ctx_create(const EmpmModelParams* params, int n_particles, int max_steps, EmpmCtx** out);
int  empm_ctx_destroy(EmpmCtx* ctx);
int  empm_ctx_set_params(EmpmCtx* ctx, const EmpmModelParams* params);

/* A batch of n_instances independent simulations advanced by the same
 * launches (the population of a CMA-ES generation, or the requests of a
 * serving slot set). Instance i has its own parameters, particle count and
 * grid; its particles occupy [poff_i, poff_i + n_particles[i]) of every
 * particle and material array passed to empm_substep / empm_rollout
 * (poff_i = sum of the previous counts), and its grid follows the previous
 * instances' grids in the grid buffers. No counterpart in the reference,
 * which evaluates a population serially (trainer_warp_mpm.py:598-661). */
int  empm_batch_create(const EmpmModelParams* params, const int* n_particles, int n_instances, int max_steps,
                       EmpmCtx** out);
int  empm_batch_set_params(EmpmCtx* ctx, int instance, const EmpmModelParams* params);

/* Grow the device buffers of a batch context to hold up to max_particles
 * particles, max_blocks 4^3 grid blocks (sum of ceil(G/4)^3 over the
 * instances) and max_instances instances. Synchronises the device: call it at
 * set-up, not while stepping. No counterpart in the reference: it serves the
 * request loop (empm_b200/serving.py), which keeps one context for a changing
 * set of requests. */
int  empm_batch_reserve(EmpmCtx* ctx, int max_particles, long long max_blocks, int max_instances);

/* Re-lay a batch context for a new set of instances within its capacity,
 * without allocating: instance i takes particles [poff_i, poff_i + n_i) in
 * order, as in empm_batch_create. The instance table is uploaded on `stream`,
 * so work of the previous layout already queued there is unaffected; work on
 * other streams that uses the context must have finished. Particle buffers
 * are the caller's: it moves the surviving instances' state to the new
 * offsets. Exceeding the capacity returns EMPM_ERR_INVALID. No counterpart in
 * the reference (it serves the request loop). */
int  empm_batch_reconfigure(EmpmCtx* ctx, const EmpmModelParams* params, const int* n_particles,
                            int n_instances, void* stream);
/* n_instances and, when non-NULL, the first particle and first grid block of each instance. */
int  empm_batch_info(EmpmCtx* ctx, int* n_instances, int* particle_offsets, int* block_offsets);

/* mu = E / (2 (1 + nu)), lam = E nu / ((1 + nu)(1 - 2 nu)); mass = density * vol,
 * written into x[4p+3]. Any of E/nu (mu/lam) or density (x) may be NULL to skip. */
int  empm_prepare(EmpmCtx* ctx, const float* E, const float* nu, float* mu, float* lam,
                  const float* density, const float* vol, float* x, int n, void* stream);

/* Reference layout <-> library layout. x3, v3: [N,3]; C9, F9: [N,3,3] row-major.
 * pack: writes x (keeps mass already in x[4p+3] when keep_mass != 0, else sets
 * it from mass3 (may be NULL -> 0)), v, C, F. NULL sources leave that plane alone. */
int  empm_pack_particles(const float* x3, const float* v3, const float* C9, const float* F9,
                         const float* mass, int keep_mass, EmpmParticles* dst, int n, void* stream);
int  empm_unpack_particles(const EmpmParticles* src, float* x3, float* v3, float* C9, float* F9,
                           int n, void* stream);

/* One MLS-MPM substep: in -> out (distinct buffers). step is a host array of
 * one schedule per instance (n_instances entries), copied to the device on
 * the given stream. */
int  empm_substep(EmpmCtx* ctx, const EmpmParticles* in, EmpmParticles* out,
                  const EmpmMaterial* mat, const EmpmStep* step, void* stream);

/* One MLS-MPM substep in place: MPMWARPDiff.p2g2p (mpm_solver_diff.py:293-429),
 * the variant of the substep whose g2p (mpm_utils.py:441-499) writes v, C and
 * F_trial back into the same state, moves x by atomic_add and then clamps it
 * (clip_particle_x, :582-599). Unsimulated particles (selection != 0) are left
 * unchanged, unlike empm_substep, where they come back cleared. The velocity
 * modifiers write the state's v in place before P2G, as there. cov: NULL, or
 * device float [n, 6] packed covariances updated with the velocity gradient
 * G as cov += dt (G cov + cov G^T) (update_cov, :306-326, applied when
 * update_cov_with_F is set). One schedule per instance, as for empm_substep. */
int  empm_substep_inplace(EmpmCtx* ctx, EmpmParticles* state, const EmpmMaterial* mat, const EmpmStep* step,
                          float* cov, void* stream);

/* n_steps substeps, ping-ponging between a and b (the result is in a when
 * n_steps is even, else in b). steps is a host array of n_tables schedule
 * tables of n_instances entries each: n_tables == 1 reuses one table for
 * every substep (static boundary conditions), n_tables == n_steps gives each
 * substep its own. With sorting enabled the particles are copied into cell
 * order inside the library at the start, re-sorted every EMPM_OPT_SORT_EVERY
 * substeps and written back in the caller's order at the end, together with
 * mu, lam, yield_stress and F_elastic. When use_graph != 0 the launch
 * sequence is captured once into a CUDA graph per (a, b, n_steps, options)
 * and replayed. */
int  empm_rollout(EmpmCtx* ctx, EmpmParticles* a, EmpmParticles* b, const EmpmMaterial* mat,
                  const EmpmStep* steps, int n_tables, int n_steps, int use_graph, void* stream);

/* empm_rollout with flags, for a rollout run as several calls (e.g. one CUDA
 * graph per block of substeps):
 *   EMPM_ROLLOUT_GRAPH   capture / replay a CUDA graph (use_graph above);
 *   EMPM_ROLLOUT_RESUME  continue from the cell-sorted state the previous
 *                        rollout on this context ended in, instead of sorting
 *                        a: the caller promises that a holds that rollout's
 *                        result, unchanged. The sort cadence continues too.
 *                        EMPM_ERR_INVALID when there is no such state (another
 *                        call re-laid, re-sorted or re-configured the context);
 *   EMPM_ROLLOUT_KEEP    leave the result in the library's sorted buffers
 *                        only: a, b and the mat arrays are not written, and a
 *                        later EMPM_ROLLOUT_RESUME call continues from it.
 * Without sorting (EMPM_OPT_SORT_EVERY 0) RESUME and KEEP have no effect.
 * Graphs are cached per launch key (buffers, n_steps, options, flags, and the
 * sorted state a resumed sequence starts in), 16 at most. */
#define EMPM_ROLLOUT_GRAPH   1
#define EMPM_ROLLOUT_RESUME  2
#define EMPM_ROLLOUT_KEEP    4
int  empm_rollout_ex(EmpmCtx* ctx, EmpmParticles* a, EmpmParticles* b, const EmpmMaterial* mat,
                     const EmpmStep* steps, int n_tables, int n_steps, int flags, void* stream);

/* Launch options of a context (empm_ctx_set_option). */
#define EMPM_OPT_SORT_EVERY  1   /* rollouts re-sort particles by 4^3 cell block every N substeps; 0 = no sorting (default 32) */
#define EMPM_OPT_P2G_MODE    2   /* sorted-path P2G: 0 = one 16-byte reduction per particle and node,
                                    1 = shared-memory node tile per chunk, 2 = warp-aggregated reductions
                                    over same-cell particles (default) */
#define EMPM_OPT_G2P_TILE    3   /* 1 = G2P stages the node tile in shared memory (default), 0 = direct gathers */
#define EMPM_OPT_TILE_CAP    4   /* nodes per shared-memory tile, 27..3072 (default 1024 = 16 KiB) */
#define EMPM_OPT_SEG_CAP     5   /* warp-aggregated P2G: same-cell runs longer than this (a power of two,
                                    1..32 lanes) are split, trading shuffle rounds for grid reductions
                                    (default 4) */
#define EMPM_OPT_ADJ_STORE   6   /* empm_adjoint_segment: 1 = keep every substep's touched grid blocks and
                                    elastic F from the segment's forward pass for the reverse pass (default;
                                    n_steps x (2 KiB per grid block + 36 B per particle) of device memory,
                                    recompute when that allocation fails); 0 = recompute P2G and the grid
                                    update in the reverse pass */
#define EMPM_OPT_FUSE        7   /* sorted rollouts with warp-aggregated P2G and direct G2P: 1 = between two cell
                                    sorts, the G2P of each substep and the stress + P2G of the next run as one
                                    kernel that keeps only position and elastic F per particle between substeps
                                    (default); 0 = separate kernels. Step tables that release a held instance
                                    (hold 1 then 0) always run separately. */
#define EMPM_OPT_SEGMENT_GRAPH 8 /* stored segments (empm_segment_forward / _reverse) and checkpointed
                                    segments (empm_adjoint_segment): 1 = their substep loops are captured as
                                    CUDA graphs on first use and replayed while the context's options and
                                    buffers are unchanged (default); 0 = launch the kernels one by one */

int  empm_ctx_set_option(EmpmCtx* ctx, int option, int value);

/* Device status word (EMPM_STATUS_* bits), read synchronously and cleared. */
int  empm_read_status(EmpmCtx* ctx, uint32_t* status, void* stream);

/* Last error message of the context (or of the library when ctx is NULL). */
int  empm_last_error(EmpmCtx* ctx, char* buf, int len);

/* One substep that allocates nothing. No counterpart in the reference.
 * For callers that cannot allocate device memory when they step the
 * simulation: for example an application that reserves all of its device
 * memory at start-up and steps the simulator inside a fixed-budget control or
 * rendering loop, where a cudaMalloc could stall or fail, or code running
 * while another framework's memory pool must not grow. The caller passes the
 * inputs and outputs as for empm_substep (particles in the caller's order,
 * one schedule for the single instance described by params; in and out share
 * no buffer). The grid scratch lives in file-scope device arrays sized for
 * grids of at most EMPM_NOALLOC_MAX_GRID^3 nodes (8 MiB, held by every GPU
 * that loads the library until the process exits); larger n_grid is rejected
 * with EMPM_ERR_INVALID. The first call on a device looks the arrays' device
 * addresses up (cudaGetSymbolAddress), so make it before any stream capture.
 * The schedule and the instance constants reach the device as kernel
 * arguments, so the call does not wait for the stream.
 * status: NULL, or a device uint32 into which the kernels OR their
 * EMPM_STATUS_* bits (NaN/Inf, CFL breach, stencil outside the grid); it is
 * not cleared by the call, so it accumulates until the caller resets it.
 * Every call in one process shares the arrays (each process that loads the
 * library has its own copy) and clears them at its start: calls that overlap
 * on the GPU (different streams or host threads of one process) race and
 * must be serialised by the caller. */
#define EMPM_NOALLOC_MAX_GRID 64
int  empm_substep_noalloc(const EmpmModelParams* params, const EmpmParticles* in, EmpmParticles* out,
                          const EmpmMaterial* mat, const EmpmStep* step, int n_particles, uint32_t* status,
                          void* stream);

/* ---- reverse mode ----------------------------------------------------------- */

/* Adjoints of the per-particle material scalars and of the mass (device
 * arrays of n_particles floats). */
typedef struct {
    float* mu;             /* in: dL/dmu after the segment; out: dL/dmu at its start */
    float* lam;            /* same for lam */
    float* yield_stress;   /* same for the yield stress */
    float* mass;           /* dL/dmass of the segment is ADDED here */
} EmpmMaterialGrad;

/* Reverse-mode differentiation of n_steps substeps starting from a
 * checkpoint. Replaces the replay of Warp's generated adjoints
 * (tape.backward, interface.py:197,418,720,935; the checkpointed replay of
 * MPMDifferentiableSimulationWCheckpoint.backward, interface.py:579-774)
 * through p2g2p_differentiable (mpm_solver_diff.py:165-291).
 *   ckpt            state at the segment start (library layout, as the input of
 *                   empm_substep; not modified);
 *   ckpt_mu/lam/yield  material scalars at the segment start (device, n floats);
 *   mat             vol and selection are used; mu, lam, yield_stress and
 *                   F_elastic are ignored;
 *   steps           n_steps tables of n_instances schedules, as given to
 *                   empm_rollout with n_tables = n_steps;
 *   grad            in: dL/d(state after the segment) in the library layout
 *                   (x and v planes as float4 with w ignored, C and F_trial as
 *                   f9 planes); out: dL/d(state at the segment start);
 *   gmat            see EmpmMaterialGrad.
 * The segment is recomputed from the checkpoint and the state of every
 * substep is kept in context-owned memory: about 120 bytes per particle and
 * substep, allocated on first use and grown as needed (so call it outside
 * stream capture). With EMPM_OPT_ADJ_STORE (the default) the re-run also
 * keeps each substep's touched grid blocks and elastic F, and the reverse pass
 * reads them; otherwise it recomputes each substep's grid first. Then the
 * three adjoint kernels run. The result is the gradient of the FP32 forward
 * map, up to FP32 rounding. The velocity written by a rotation modifier is
 * treated as independent of x. With EMPM_OPT_SEGMENT_GRAPH the re-run and the
 * reverse pass are captured as a CUDA graph, cached in the context (a few
 * entries, by segment length and options), and replayed by later calls with
 * the same key. */
int  empm_adjoint_segment(EmpmCtx* ctx, const EmpmParticles* ckpt, const float* ckpt_mu, const float* ckpt_lam,
                          const float* ckpt_yield, const EmpmMaterial* mat, const EmpmStep* steps, int n_steps,
                          EmpmParticles* grad, EmpmMaterialGrad* gmat, void* stream);

/* Stored segments: the forward pass of a differentiable rollout keeps, per
 * segment, everything its reverse pass reads, so that the reverse pass does
 * not recompute the segment from a checkpoint. This is what Warp's tape does
 * for the reference (MyTape records every launch of p2g2p_differentiable,
 * warp_utils.py:93-127, interface.py:135-145, and tape.backward replays the
 * adjoints, interface.py:197); here a segment keeps about
 * 152 B per particle and substep + 2 KiB per touched grid block and substep,
 * and empm_segment_bytes gives the exact figure.
 *
 * empm_segment_create   allocates the store for n_steps substeps of the
 *                       context's current particle count, with room for
 *                       block_cap touched grid blocks per substep (0: every
 *                       block of the context's grids); EMPM_ERR_OOM (nothing
 *                       left allocated) when it does not fit. Call it outside
 *                       stream capture.
 * empm_segment_forward  runs n_steps substeps from ckpt / ckpt_mu / ckpt_lam /
 *                       ckpt_yield (not modified) as empm_rollout would, keeping
 *                       the store. The state after the last substep goes to
 *                       out (library layout); mat->mu, lam, yield_stress and
 *                       F_elastic receive the updated values (they may alias the
 *                       ckpt_* arrays); mat->vol and selection are read. Steps:
 *                       n_steps tables of n_instances schedules.
 * empm_segment_blocks   waits for the stream and gives the largest number of
 *                       grid blocks any substep of the last forward pass
 *                       touched, and the segment's block_cap. Over block_cap,
 *                       that forward pass could not keep its grids: make a
 *                       segment with a larger block_cap and run it again.
 * empm_segment_reverse  the adjoint of that forward pass: grad holds
 *                       dL/d(out) on entry and dL/d(ckpt) on return; gmat as for
 *                       empm_adjoint_segment. The context's model parameters
 *                       must still be those of the forward pass. A segment may
 *                       be reversed more than once. It checks the touched
 *                       block count (empm_segment_blocks, once per forward
 *                       pass) and returns EMPM_ERR_INVALID after an overflow.
 * A segment keeps a device copy of its step tables (uploaded again only when
 * they change) and, with EMPM_OPT_SEGMENT_GRAPH, its captured substep loops:
 * the first forward and reverse pass of a segment capture them, so make those
 * calls outside stream capture.
 * Gradients equal those of empm_adjoint_segment (which stores and reverses one
 * segment inside one call) up to the order of floating-point reductions. */
typedef struct EmpmSegment EmpmSegment;
int  empm_segment_bytes(EmpmCtx* ctx, int n_steps, int block_cap, size_t* out);
int  empm_segment_create(EmpmCtx* ctx, int n_steps, int block_cap, EmpmSegment** out);
int  empm_segment_blocks(EmpmSegment* seg, int* max_touched, int* block_cap, void* stream);
int  empm_segment_destroy(EmpmSegment* seg);
int  empm_segment_forward(EmpmCtx* ctx, EmpmSegment* seg, const EmpmParticles* ckpt, const float* ckpt_mu,
                          const float* ckpt_lam, const float* ckpt_yield, const EmpmMaterial* mat,
                          const EmpmStep* steps, int n_steps, EmpmParticles* out, void* stream);
int  empm_segment_reverse(EmpmCtx* ctx, EmpmSegment* seg, EmpmParticles* grad, EmpmMaterialGrad* gmat,
                          void* stream);

/* Chain rule through empm_prepare: dL/dE and dL/dnu from dL/dmu and dL/dlam
 * (compute_mu_lam_from_E_nu, mpm_utils.py:277-283), and dL/ddensity =
 * dL/dmass * vol (get_float_array_product, mpm_data_structure.py:719-726).
 * Either group of pointers may be NULL. */
int  empm_prepare_adjoint(const float* E, const float* nu, const float* g_mu, const float* g_lam, float* g_E,
                          float* g_nu, const float* vol, const float* g_mass, float* g_density, int n, void* stream);

/* Static-pose restart: replaces MPMWARPDiff.restart_and_compute_F_C
 * (mpm_solver_diff.py:1214-1262; kernels set_F_C_p2g / set_F_C_g2p,
 * mpm_utils.py:836-919). The displacement target - x of every simulated
 * particle is scattered to its instance's grid with weight * mass, normalised
 * by the grid mass (no gravity, no boundary conditions), and gathered back as
 * F_trial = I + sum grid_v (x) dweight. Then every particle's x becomes its
 * target (float [n, 3]); C is unchanged. selection: NULL or device int [n]
 * (non-zero: F_trial kept). cov: NULL, or device float [n, 6] packed
 * covariances (c00, c01, c02, c11, c12, c22) updated as cov += G cov + cov G^T
 * with G = F_trial - I, the PhysGaussian update the reference applies here
 * when update_cov_with_F is set (update_cov, mpm_utils.py:306-326, :918-919). */
int  empm_restart_F(EmpmCtx* ctx, EmpmParticles* particles, const float* target, const int* selection, float* cov,
                    void* stream);

/* ---- training losses --------------------------------------------------------- */

/* Chamfer distance of many point-set pairs in one launch, the loss of the
 * reference trainer (pytorch3d chamfer_distance with point_reduction "mean",
 * phys_sim/engine/trainer_warp_mpm.py:542-561,617-642,745-765). Pair p owns
 * rows [x_off[p], x_off[p+1]) of x and [y_off[p], y_off[p+1]) of y (device
 * int arrays of n_pairs + 1 entries; x, y: [rows, 3] floats). Returns, per
 * pair, sum_xy[p] = sum over x of min_y |x - y|^2 and sum_yx[p] likewise; the
 * chamfer distance is sum_xy / nx_p + sum_yx / ny_p. nn_x / nn_y receive the
 * index (row of the other set) of each point's nearest neighbour, for the
 * gradient. max_nx / max_ny: the largest set size of any pair (launch shape).
 * Exact brute force over shared-memory tiles. */
int  empm_chamfer(const float* x, const int* x_off, int nx, int max_nx, const float* y, const int* y_off, int ny,
                  int max_ny, int n_pairs, float* sum_xy, float* sum_yx, int* nn_x, int* nn_y, void* stream);

/* Gradient in x of sum_p (g_xy[p] * sum_xy[p] + g_yx[p] * sum_yx[p]) for the
 * neighbours found by empm_chamfer, ADDED to grad_x ([nx, 3]). scratch_pair:
 * device int array of max(nx, ny) entries. */
int  empm_chamfer_backward(const float* x, const int* x_off, int nx, const float* y, const int* y_off, int ny,
                           int n_pairs, const int* nn_x, const int* nn_y, const float* g_xy, const float* g_yx,
                           float* grad_x, int* scratch_pair, void* stream);

/* ---- Gaussian motion interpolation (linear blend skinning) ------------------ */

/* Per-frame transfer of the simulated particle motion to the rendered
 * Gaussians, third_party/gaussian_splatting/dynamic_utils.py. Index arrays
 * (relations, neighbour indices) are [rows, k] of int64 (idx_bytes 8, what
 * torch.topk returns) or int32 (idx_bytes 4). Indices outside [0, n_bones)
 * are not read: the affected outputs become NaN and bit 1 of *status (device
 * int, or counts[EMPM_LBS_STATUS]) is set; the reference's indexing raises. */
#define EMPM_KNN_MAX_K     32
#define EMPM_QUAT_KORNIA   0   /* kornia 0.8.1 rotation_matrix_to_quaternion (dynamic_utils.py:465-475) */
#define EMPM_QUAT_MAT2QUAT 1   /* mat2quat, dynamic_utils.py:25-64 */
#define EMPM_LBS_COUNTS    8   /* ints of the counts array of empm_lbs_bones */
#define EMPM_LBS_STATUS    6   /* counts[EMPM_LBS_STATUS]: status bits of the bone stage */
#define EMPM_LBS_TABLE_FLOATS 16   /* floats per bone of the bone table */

/* Exact k nearest neighbours (k <= EMPM_KNN_MAX_K): for every query row, the
 * k rows of points closest to it, nearest first, equal distances in index
 * order. exclude_self != 0 (queries == points) leaves each point out of its
 * own list. Replaces get_topk_indices (dynamic_utils.py:248-265: topk of K+1
 * with the first dropped) and the search of knn_weights_sparse (:295-302).
 * out_dist (optional): the Euclidean distances. */
int  empm_knn(const float* queries, int n_queries, const float* points, int n_points, int k, int exclude_self,
              void* out_idx, int idx_bytes, float* out_dist, void* stream);

/* Inverse-distance weights of the k given bones of every point:
 * w = 1 / (|x - b| + 1e-6), normalised over the k
 * (calc_weights_vals_from_indices, dynamic_utils.py:282-292). */
int  empm_idw_weights(const float* bones, int n_bones, const float* pts, int n, const void* idx, int idx_bytes,
                      int k, float* weights, int* status, void* stream);

/* Bone stage of interpolate_motions(_speedup) (dynamic_utils.py:315-409):
 * per bone the rotation fitted to its n_adj neighbours' motion, resolved over
 * all bones as the reference assigns them, and its unit quaternion in the
 * given convention. Writes table [n_bones * EMPM_LBS_TABLE_FLOATS] (32-byte
 * aligned) and uses work [n_bones * 10] floats and counts [EMPM_LBS_COUNTS]
 * ints (device; counts[0..2] = bones of rank 0, 1, 2-3). */
int  empm_lbs_bones(const float* bones, const float* motions, int n_bones, const void* relations, int idx_bytes,
                    int n_adj, int convention, float* table, float* work, int* counts, void* stream);

/* Gaussian stage of interpolate_motions_speedup (dynamic_utils.py:428-483):
 * xyz_out = sum_k w (R (x - b) + m + b) over the k bones of each Gaussian;
 * quat_out = normalize(sum_k w q_bone) * quat_in ((w, x, y, z); skipped when
 * quat_in is NULL). weights NULL: the weights of empm_idw_weights for the
 * table's bones, computed in the same pass (and written to weights_out when
 * given), as the reference's per-frame loop recomputes them before the call
 * (trainer_warp_mpm.py:1644-1655). Outputs may alias the inputs. */
int  empm_lbs_blend(const float* table, int n_bones, const float* xyz, const float* quat_in, int n, const void* idx,
                    int idx_bytes, int k, const float* weights, float* weights_out, float* xyz_out, float* quat_out,
                    int* status, void* stream);

/* Gaussian stage of interpolate_motions (dynamic_utils.py:165-216) with
 * dense [n, n_bones] weights; weights NULL: inverse distance to every bone,
 * 1 / max(d, 1e-4) normalised, also written to weights_out when given. */
int  empm_lbs_blend_dense(const float* table, int n_bones, const float* xyz, const float* quat_in, int n,
                          const float* weights, float* weights_out, float* xyz_out, float* quat_out, void* stream);

/* Quaternions (w, x, y, z) of n row-major rotation matrices, unnormalised,
 * in the given convention (mat2quat, dynamic_utils.py:25-64, or kornia's). */
int  empm_rotation_to_quat(const float* R9, int n, int convention, float* q, void* stream);

/* ---- diagnostics (used by the parity tests) ------------------------------ */

/* Adjoint of empm_debug_stress for n particles (row-major [N,3,3] like it):
 * given dL/dF_elastic, dL/dstress and dL/d(mu, lam, yield after the update),
 * returns dL/dF_trial and overwrites g_mu, g_lam, g_yield with dL/d(mu, lam,
 * yield before the update). mu, lam, yield_stress are inputs only. */
int  empm_debug_stress_adjoint(const EmpmModelParams* params, const float* F_trial9, const float* mu,
                               const float* lam, const float* yield_stress, float dt, const float* g_F9,
                               const float* g_stress9, float* g_mu, float* g_lam, float* g_yield,
                               float* g_F_trial9, int n, void* stream);

/* Return map + Kirchhoff stress of the material switch for n particles, on
 * the device, in the reference's [N,3,3] row-major layout: the body of
 * compute_stress_from_F_trial (mpm_utils.py:602-665). mu, lam, yield_stress
 * are updated in place as the reference's return maps do. */
int  empm_debug_stress(const EmpmModelParams* params, const float* F_trial9, float* mu, float* lam,
                       float* yield_stress, float dt, float* F_out9, float* stress_out9, int n, void* stream);

/* Per-kernel timing with CUDA events on the launch stream (stream path of
 * empm_substep / empm_rollout only; graph replays are not instrumented).
 * enable != 0 starts a fresh measurement with room for max_launches launches
 * per kernel; empm_ctx_kernel_times synchronises and returns, for the three
 * kernels of a substep [stress+P2G, grid update, G2P], the summed duration in
 * milliseconds and the number of launches timed. */
int  empm_ctx_timing(EmpmCtx* ctx, int enable, int max_launches);
int  empm_ctx_kernel_times(EmpmCtx* ctx, float* total_ms3, int* launches3);
/* The same for the three adjoint kernels of empm_adjoint_segment: adjoint
 * G2P, adjoint grid update, adjoint P2G (the recomputed forward P2G and grid
 * update of the adjoint are counted with the forward kernels). */
int  empm_ctx_adjoint_kernel_times(EmpmCtx* ctx, float* total_ms3, int* launches3);
/* The same for the fused G2P + stress + P2G kernel of EMPM_OPT_FUSE rollouts
 * (the runs' first stress + P2G and last G2P are counted with the separate
 * kernels above). */
int  empm_ctx_fused_kernel_times(EmpmCtx* ctx, float* total_ms, int* launches);

/* Device pointers of the context's grid buffers: float4 per node in the
 * blocked layout (4x4x4-node blocks of 64 consecutive float4, block (bi,bj,bk)
 * at (bi*NB + bj)*NB + bk with NB = ceil(G/4), node (i&3,j&3,k&3) at
 * (i&3)*16 + (j&3)*4 + (k&3) inside it): the P2G accumulator (zero between
 * substeps) and the node velocities of the last grid update (w = node mass).
 * Only nodes of blocks touched by the last substep's particles are current. */
int  empm_ctx_grid(EmpmCtx* ctx, float** momentum, float** velocity);

#ifdef __cplusplus
}
#endif
#endif /* EMPM_B200_H */
