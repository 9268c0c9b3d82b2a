/*
 * vxp.h — C ABI of the B200 voxel contact-generation + TGS-soft solver library.
 *
 * This header is the drop-in boundary for the per-step hot path of the Zig
 * engine nitanmarcel/zig-voxel-physics.  In that engine the seams are two
 * concrete structs held by value in VoxelPhysicsSystem (src/system.zig:195-198):
 *
 *   narrow_phase: NarrowPhase   — beginFrame / processPair / getContactManager
 *   solver:       ContactSolver — clear / addBody / setContactManager /
 *                                 addManifold / solve
 *
 * and the frame entry VoxelPhysicsSystem.step (src/system.zig:537-555), which
 * runs narrowPhase() (src/system.zig:586-655), solve() (src/system.zig:670-783)
 * and updateSleepStates() (src/system.zig:786-792) once per fixed step.  The
 * entry points below replace those calls; the broad phase stays with the host
 * and hands its pair list across (BodyPair, src/broad_phase.zig:17-39).
 *
 * Conventions
 *   - Every function returns an int status: VXP_OK (0) or a negative VXP_ERR_*.
 *     vxp_last_error() gives a one-line message for the last failing call.
 *   - The context owns all device memory.  Host buffers are borrowed for the
 *     duration of the call only.
 *   - One host thread and one CUDA stream per context.
 *   - All layouts are plain C structs with fixed-width fields (no padding
 *     surprises: every struct is a multiple of 4 bytes and only the manifold
 *     contact carries a u64, placed 8-byte aligned).
 */
#ifndef VXP_H
#define VXP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VXP_ABI_VERSION 2

/* ---- status codes (Zig error unions swallowed by `catch {}` in the
 *      reference become explicit codes here; src/system.zig:577,610,637,...) */
#define VXP_OK            0
#define VXP_ERR_ARG      -1  /* bad argument, unknown id, size mismatch      */
#define VXP_ERR_OOM      -2  /* device or host allocation failed             */
#define VXP_ERR_CUDA     -3  /* a CUDA runtime call failed                   */
#define VXP_ERR_TIMEOUT  -4  /* a bounded device-side wait ran out           */
#define VXP_ERR_CAP      -5  /* a configured capacity was exceeded           */
#define VXP_ERR_STATE    -6  /* call out of order (e.g. no colliders)        */

/* ---- body types (BodyType, src/body.zig:29-48) */
#define VXP_BODY_STATIC    0u
#define VXP_BODY_KINEMATIC 1u
#define VXP_BODY_DYNAMIC   2u

/* ---- solver constraint ordering.  The reference sweeps manifolds in
 *      ContactManager hash-map order (src/solver.zig:733); a parallel sweep
 *      needs colour batches.  Both modes order the sweep colour-major.      */
#define VXP_COLOUR_PROJECT   0u  /* greedy over writable (dynamic, awake) bodies,
                                    Jones-Plassmann priorities              */
#define VXP_COLOUR_REFERENCE 1u  /* GraphColoring.build (src/islands.zig:668-736):
                                    first-fit in manifold order, every body a node */

/* One 8x8x8 brick of CollisionVoxel bytes (CollisionBrick.voxels,
 * src/collider.zig:44-46): index x + 8*y + 64*z; bits 0-2 = VoxelType,
 * bits 3-7 = NORMAL_LUT index (packed struct, src/collision_voxel.zig:133-140). */
typedef struct {
    int32_t pos[3];        /* brick position in brick coordinates */
    uint8_t voxels[512];
} vxp_brick;               /* 524 bytes */

/* VoxelBody (src/body.zig:177-203) flattened: BodyMotionState + BodyProperties
 * + sleep fields + the collider it references. */
typedef struct {
    uint32_t id;                 /* unique, > 0; the smaller id is body A   */
    uint32_t body_type;          /* VXP_BODY_*                              */
    uint32_t collider_id;        /* as passed to vxp_collider_upload        */
    uint32_t is_sleeping;        /* 0/1                                     */
    float position[3];
    float rotation[4];           /* quaternion x, y, z, w                   */
    float linear_velocity[3];
    float angular_velocity[3];
    float inv_mass;
    float inv_inertia_local[9];  /* Mat3 m[i][j] row-major                  */
    float friction;
    float restitution;
    float linear_damping;
    float angular_damping;
    float sleep_timer;
} vxp_body;                      /* 32 x 4 = 128 bytes */

/* BodyPair (src/broad_phase.zig:17-28); body_a < body_b. */
typedef struct {
    uint32_t body_a;
    uint32_t body_b;
} vxp_pair;

/* ContactPoint (src/narrow_phase.zig:336-393) in field order. */
typedef struct {
    float point[3];
    float normal[3];
    float penetration;
    float local_anchor_a[3];
    float local_anchor_b[3];
    float normal_impulse;
    float tangent_impulse[2];
    float normal_mass;
    float tangent_mass[2];
    uint32_t _pad;
    uint64_t feature_id;
} vxp_contact;                   /* 88 bytes */

/* ContactManifold (src/narrow_phase.zig:416-448); friction_anchor is never
 * set by the reference and is omitted. */
typedef struct {
    uint32_t body_a_id;
    uint32_t body_b_id;
    uint32_t contact_count;
    float friction;
    float restitution;
    uint32_t _pad;
    vxp_contact contacts[4];
} vxp_manifold;                  /* 24 + 352 = 376 bytes */

/* PhysicsConfig (src/system.zig:47-88) + SolverConfig (src/solver.zig:75-119)
 * + NarrowPhaseConfig (src/narrow_phase.zig:1325-1343) + the two documented
 * deviation flags.  vxp_config_default() fills the reference defaults. */
typedef struct {
    /* PhysicsConfig */
    float gravity[3];
    float fixed_timestep;
    uint32_t enable_sleeping;
    uint32_t enable_warm_starting;
    /* SolverConfig */
    uint32_t substeps;
    uint32_t velocity_iterations;
    uint32_t position_iterations;
    uint32_t disable_rotation;
    float hertz;
    float damping_ratio;
    float position_correction_rate;
    float max_position_correction;
    float slop;
    uint32_t warm_starting;
    float warm_start_scale;
    uint32_t enable_friction;
    uint32_t enable_restitution;
    /* NarrowPhaseConfig */
    uint32_t use_brick_sat;
    uint32_t use_brick_pair_cache;
    uint32_t brick_pair_cache_size;
    /* deviation flags */
    uint32_t reference_caps;     /* 1: keep the reference's 512-pair cap
                                    (src/system.zig:594,612); 0: uncapped   */
    uint32_t colouring;          /* VXP_COLOUR_*                           */
    uint32_t enable_islands;     /* PhysicsConfig.enable_islands: IslandManager
                                    statistics each solve (system.zig:705-760) */
    /* capacities (device buffers are sized from these; 0 = grow on demand) */
    uint32_t max_bodies;
    uint32_t max_pairs;
} vxp_config;

/* Per-step counters: NarrowPhase.stats (src/narrow_phase.zig:1355-1366) and
 * SolverStats (src/solver.zig:381-392), plus device-side extras. */
typedef struct {
    uint32_t pairs_in;               /* pairs handed in                      */
    uint32_t pairs_tested;           /* processPair calls                    */
    uint32_t pairs_colliding;
    uint32_t voxels_checked;
    uint32_t contacts_generated;
    uint32_t pairs_skipped_sleeping; /* system-level + narrow-phase skips    */
    uint32_t manifolds_preserved;
    uint32_t cache_hits;
    uint32_t cache_misses;
    uint32_t cache_evictions;
    uint32_t manifolds;              /* manifolds in the ContactManager      */
    uint32_t constraints;            /* manifolds handed to the solver       */
    uint32_t contact_points;         /* points in the solver's constraint set*/
    uint32_t colours;                /* colour batches used by the sweep     */
    uint32_t position_iterations_run;
    uint32_t step_skipped;           /* 1 when every dynamic body slept      */
    float max_penetration;
    uint32_t candidates;             /* distance-passing voxel pairs         */
    uint32_t bricks_touched;         /* bricks of A inside the overlap region
                                        plus bricks of B inside B's, summed over
                                        the pairs detected (traffic accounting) */
    uint32_t sweep_path;             /* how the solver's sweeps ran on the
                                        thread-block cluster: 1 every constraint
                                        row in shared memory, 2 the rows that did
                                        not fit in global memory, 3 all state in
                                        L2; 0 no cluster sweep this step      */
    /* PhysicsStats island fields (src/system.zig:119-122), from the
     * IslandManager after this step's build and sleep update; 0 when islands
     * are off or the step was skipped */
    uint32_t island_count;
    uint32_t active_islands;
    uint32_t sleeping_islands;
    uint32_t largest_island_size;
} vxp_stats;

/* One candidate voxel pair of the narrow phase, for parity checks of the
 * candidate set (checkNeighborhood, src/narrow_phase.zig:796-857). */
typedef struct {
    uint32_t pair_index;   /* index into the pair list handed in            */
    int32_t a[3];          /* voxel of body A                               */
    int32_t b[3];          /* voxel of body B                               */
    uint32_t passed;       /* 1: dist^2 < speculative threshold             */
    float dist_sq;
} vxp_candidate;           /* 36 bytes */

typedef struct vxp_ctx vxp_ctx;

/* ---------------------------------------------------------------------------
 * Context
 * ------------------------------------------------------------------------- */

/* Reference defaults: PhysicsConfig{} + SolverConfig{} + NarrowPhaseConfig{}. */
void vxp_config_default(vxp_config* cfg);

/* Replaces VoxelPhysicsSystem.init's NarrowPhase.init / ContactSolver.init
 * (src/system.zig:248-249).  device = CUDA ordinal. */
int vxp_create(const vxp_config* cfg, int device, vxp_ctx** out);
void vxp_destroy(vxp_ctx* ctx);
int vxp_last_error(const vxp_ctx* ctx, char* buf, size_t n);
int vxp_abi_version(void);

/* ---------------------------------------------------------------------------
 * Colliders and bodies
 * ------------------------------------------------------------------------- */

/* Uploads one VoxelCollider (src/collider.zig:144-409): its bricks and voxel
 * size.  Bounds, local AABB and solid count are recomputed as
 * VoxelCollider.recomputeMetadata does (src/collider.zig:283-333).
 * Bricks whose hashBrickPos collide (src/collider.zig:187-192) are rejected. */
int vxp_collider_upload(vxp_ctx* ctx, uint32_t collider_id, float voxel_size,
                        const vxp_brick* bricks, uint32_t n_bricks);

/* Collider edits, for destructible or growing voxel bodies.  An edit batch
 * writes n voxels of an uploaded collider (coords: 3 ints per voxel, in the
 * collider's voxel space) and then does what the reference's caller does
 * after setCollisionVoxel (src/collider.zig:267-273): recomputeMetadata
 * (src/collider.zig:283-333).  Modes:
 *   VXP_EDIT_SET        values[i] is the CollisionVoxel byte stored
 *                       (src/collision_voxel.zig:133-167: type in bits 0-2,
 *                       normal index in bits 3-7), as setCollisionVoxel stores it;
 *   VXP_EDIT_OCCUPANCY  values[i] != 0 makes the voxel solid, 0 empty; then
 *                       every listed voxel and each of its six face
 *                       neighbours that is solid is re-typed by
 *                       classifyFromNeighbors (src/collision_voxel.zig:213-235,
 *                       exported by src/physics.zig:52) of the new occupancy.
 * Writes run in list order (a voxel listed twice keeps its last value).  A
 * voxel whose brick the collider lacks gets a new brick, as getOrCreateBrick
 * (src/collider.zig:232-239) makes one, in the order the writes reach them.
 * The edit is queued on the context's stream after the steps already queued,
 * and the next step sees it; the bodies' collider ids are unchanged.  Cached
 * brick-pair results of the bodies that use the collider stay valid until
 * vxp_invalidate_cache_for_body drops them, as in the reference. */
#define VXP_EDIT_SET 0
#define VXP_EDIT_OCCUPANCY 1
int vxp_collider_edit(vxp_ctx* ctx, uint32_t collider_id, const int32_t* coords,
                      const uint8_t* values, uint32_t n, int mode);

/* The collider as the device holds it: metadata, and up to cap bricks (in
 * the collider's brick order: uploaded bricks first, then those that edits
 * created).  *n_bricks gets the collider's brick count.  bricks may be null. */
typedef struct vxp_collider_info {
    float voxel_size;
    int32_t min_bound[3], max_bound[3];  /* voxel coordinates, max exclusive */
    float aabb_min[3], aabb_max[3];      /* local AABB */
    uint32_t solid_count;
    uint32_t n_bricks;
    uint32_t has_table;                  /* the probes use a neighbourhood-mask table */
} vxp_collider_info;
int vxp_collider_read(vxp_ctx* ctx, uint32_t collider_id, vxp_collider_info* info,
                      vxp_brick* bricks, uint32_t cap, uint32_t* n_bricks);

/* NarrowPhase.invalidateCacheForBody (src/narrow_phase.zig:1399-1403): every
 * brick-pair cache entry of the body becomes invalid.  *n_invalidated (may be
 * null; when given, the call waits for the device) gets their number, the
 * cache's invalidations statistic (src/narrow_phase.zig:305-312). */
int vxp_invalidate_cache_for_body(vxp_ctx* ctx, uint32_t body_id, uint32_t* n_invalidated);

/* Replaces the per-slot body state that step() reads and writes.  Bodies are
 * kept in the order given (the solver's addBody order, src/system.zig:677-681). */
int vxp_bodies_set(vxp_ctx* ctx, const vxp_body* bodies, uint32_t n);
int vxp_bodies_get(vxp_ctx* ctx, vxp_body* bodies, uint32_t n);

/* Bulk state export for a renderer or another CUDA consumer: the per-handle
 * getters getPosition, getRotation, getLinearVelocity, getAngularVelocity,
 * getWorldAABB and isSleeping (src/system.zig:963-1017; getWorldAABB is the
 * collider's local AABB through AABB.transform, src/body.zig:430-435,
 * src/collider.zig:341-343, src/math.zig:686-693) for bodies
 * [first, first + n) in vxp_bodies_set order, one array per field.  Every
 * null pointer is skipped.  Layouts: 3 floats a body (x, y, z) for vectors,
 * 4 for the rotation (x, y, z, w), one byte for sleeping (1 = asleep). */
typedef struct {
    float* position;
    float* rotation;
    float* linear_velocity;
    float* angular_velocity;
    float* aabb_min;
    float* aabb_max;
    uint8_t* sleeping;
} vxp_state_view;

/* device_memory = 0: the pointers are host memory (pinned is faster); the
 * call returns once they are filled.
 * device_memory = 1: every pointer is device memory of the context's device
 * (checked; anything else is VXP_ERR_ARG), e.g. an instance buffer that a
 * renderer maps for CUDA.  One kernel writes them on the context's stream
 * after the work already queued there, and the call returns without waiting.
 * When consumer_stream (a cudaStream_t) is not null, that stream waits for
 * the export, so whatever the caller launches there next reads the state. */
int vxp_bodies_export(vxp_ctx* ctx, const vxp_state_view* dst, uint32_t first, uint32_t n, int device_memory,
                      void* consumer_stream);

/* Host-side computeMassProperties (src/body.zig:462-519) over a brick list in
 * the order given; the inertia sum runs brick by brick, voxel index order. */
int vxp_mass_properties(float voxel_size, const vxp_brick* bricks, uint32_t n_bricks,
                        float density, float* inv_mass, float inv_inertia[9]);

/* ---------------------------------------------------------------------------
 * The per-step hot path
 * ------------------------------------------------------------------------- */

/* One VoxelPhysicsSystem.step (src/system.zig:537-555) with the broad-phase
 * pairs given: narrowPhase + solve + updateSleepStates, all on the device. */
int vxp_step(vxp_ctx* ctx, float dt, const vxp_pair* pairs, uint32_t n_pairs);

/* Same step, with the pair list produced on the device from inflated world
 * AABBs (margin in metres) instead of handed in. */
int vxp_step_device_pairs(vxp_ctx* ctx, float dt, float margin);

/* The two halves of the step, for tests: narrowPhase() then solve()+sleep. */
int vxp_narrow_phase(vxp_ctx* ctx, const vxp_pair* pairs, uint32_t n_pairs);
int vxp_solve(vxp_ctx* ctx, float dt);

/* ContactManager.manifolds after the last narrow phase, in manifold order
 * (pair order).  *n_out = number written (<= cap). */
int vxp_manifolds_get(vxp_ctx* ctx, vxp_manifold* out, uint32_t cap, uint32_t* n_out);

/* Every type-filter-passing voxel pair of the last narrow phase (debug mode:
 * enable with vxp_set_candidate_dump before vxp_narrow_phase). */
int vxp_set_candidate_dump(vxp_ctx* ctx, uint32_t capacity);
int vxp_candidates_get(vxp_ctx* ctx, vxp_candidate* out, uint32_t cap, uint32_t* n_out);

int vxp_stats_get(vxp_ctx* ctx, vxp_stats* out);

/* Colours of the last solve, indexed like the constraint list. */
int vxp_colours_get(vxp_ctx* ctx, uint32_t* colours, uint32_t cap, uint32_t* n_out);

/* Pair source used by tests, the bench and vxp_step_device_pairs: every
 * (min id, max id) pair, not both static, whose world AABBs inflated by
 * margin overlap, sorted by (body_a, body_b).  Computed on the device from the
 * current body state. */
int vxp_pairs_from_bodies(vxp_ctx* ctx, float margin, vxp_pair* out, uint32_t cap,
                          uint32_t* n_out);

/* Device time of the last step call (ms, CUDA events on the context's
 * stream): [pair source and copies, step kernel, whole call]. */
int vxp_last_step_ms(vxp_ctx* ctx, float out[3]);

/* Per-substep parity hook.  With recording on, each step writes every body's
 * state after each substep's relax sweep (BodyState after relaxConstraints,
 * src/solver.zig:848-856; before the position sweeps and writeBack) as 13
 * floats: position[3], rotation[4], linear_velocity[3], angular_velocity[3],
 * substep-major, bodies in vxp_bodies_set order.  Recording steps sweep colour
 * batch by colour batch (bit-identical to the event-ordered sweeps).
 * vxp_substeps_get waits for the last step; *n_substeps = substeps recorded
 * (0 when the step was skipped); cap_floats must hold n_substeps x bodies x 13. */
int vxp_snapshot_substeps(vxp_ctx* ctx, int enable);
int vxp_substeps_get(vxp_ctx* ctx, float* out, uint32_t cap_floats, uint32_t* n_substeps);

/* Device time (ms) of the last step's kernels: [narrow part, solve part].  A
 * world stepped by the cooperative grid runs them as two kernels
 * (k_step_grid, k_solve_grid); a world stepped by one CTA runs both parts in
 * one kernel, reported in out[0] with out[1] = 0. */
int vxp_last_kernel_ms(vxp_ctx* ctx, float out[2]);

/* Step calls queue work on the context's stream and return; a call that
 * returns data (bodies, manifolds, stats, colours, candidates) waits for it.
 * vxp_synchronize waits without copying and reports any device-side error
 * (VXP_ERR_TIMEOUT, VXP_ERR_CAP) of the steps queued since the last wait.
 * VXP_ERR_CAP from a step means the step left all state untouched: grow the
 * capacity (vxp_config.max_pairs) and run it again. */
int vxp_synchronize(vxp_ctx* ctx);

/* -1: choose per step (default); 0: one CTA steps the world; 1: the world is
 * stepped by a cooperative grid over every SM. */
int vxp_set_launch_mode(vxp_ctx* ctx, int mode);

/* Grid launch tuning: after the narrow phase, the solver runs on
 * ceil(manifolds / div) blocks (at least 2); default div 128. */
int vxp_set_solver_blocks_divisor(vxp_ctx* ctx, uint32_t div);

/* Narrow-phase work split: a pair whose overlap region holds at least n
 * voxels is probed by a whole CTA before the other pairs, which are probed one
 * warp each (default 2048; 0: every pair by one warp; the worlds of a batch,
 * one CTA each, use 1024).  Results do not depend on it. */
int vxp_set_heavy_pair_voxels(vxp_ctx* ctx, uint32_t n);

/* Narrow-phase probe tables: with enable (the default) every collider of at
 * most 2^23 probe centres gets a table of its voxels' 27-neighbour type masks
 * when the colliders upload, and a probe centre costs one lookup instead of
 * 27; with 0 every probe looks its voxels up.  Takes effect at the next step.
 * Results do not depend on it. */
int vxp_set_probe_tables(vxp_ctx* ctx, int enable);

/* Longest time a block of a grid-launched step waits at a grid barrier
 * before the step gives up with VXP_ERR_TIMEOUT (0: the default, 10 s).  A
 * failure-detection knob: a limit of a few nanoseconds makes a real step run
 * out at its first uneven barrier, the kernels return, the call reports
 * VXP_ERR_TIMEOUT and the context keeps working.  No counterpart in the
 * reference, which has no bounded waits. */
int vxp_set_wait_limit_ns(vxp_ctx* ctx, uint64_t ns);

/* Order of the solver's sweeps (ContactSolver.solve, src/solver.zig:494-561)
 * when a world is stepped by the cooperative grid (vxp_set_launch_mode).
 * 2 (default where the device schedules the cluster, see vxp_cluster_size):
 * the constraints and colouring on the grid, then the sweeps and the store on
 * one thread-block cluster (16 CTAs, or 8) with a hardware cluster barrier
 * after every colour batch and the bodies and constraint rows in the
 * cluster's shared memory (in L2 when they do not fit); 1 (the default
 * otherwise): each manifold waits only for the earlier manifolds of its own
 * two bodies (per-body event counters), so colour batches and sweeps overlap;
 * 0: a software grid barrier after every colour batch.  All give
 * bit-identical results; a step with a kinematic body in a constraint uses 0
 * under mode 1, and every world stepped by a single CTA (small worlds,
 * batches) sweeps with CTA barriers.  Mode 2 where no cluster can be
 * scheduled returns VXP_ERR_STATE. */
#define VXP_SOLVER_BARRIERS 0u
#define VXP_SOLVER_EVENTS 1u
#define VXP_SOLVER_CLUSTER 2u
int vxp_set_solver_mode(vxp_ctx* ctx, uint32_t mode);

/* CTAs of the cluster that mode VXP_SOLVER_CLUSTER runs on (0: none). */
int vxp_cluster_size(vxp_ctx* ctx, uint32_t* n);

/* Shared memory (bytes per CTA) that the cluster's sweeps may hold their state
 * in: the bodies and the velocity-sweep fields of the constraint rows.  A step
 * whose state does not fit sweeps with that state in L2 instead (same
 * results).  Default: all a block can have; 0: always in L2. */
int vxp_set_cluster_shared_bytes(vxp_ctx* ctx, uint32_t bytes);

/* Traffic accounting: with on, each step counts the voxel bricks its probed
 * pairs touch (vxp_stats.bricks_touched: A's bricks in the overlap region plus
 * B's bricks in B's region), for the narrow phase's algorithmic-byte figure.
 * It costs time in the narrow phase, so it is off by default (the count reads
 * 0); results do not depend on it. */
int vxp_set_traffic_accounting(vxp_ctx* ctx, int on);

/* Under VXP_SOLVER_CLUSTER: 0 (default) the grid builds the constraint table
 * and colours it (k_solve_grid), then the cluster sweeps; 1 the cluster does
 * all of the solve part (one kernel; slower on large worlds, where the
 * colouring wants more SMs).  Same results. */
int vxp_set_cluster_constraints(vxp_ctx* ctx, int on);

/* Device time (ms) of the last step's solve part split by kernel under
 * VXP_SOLVER_CLUSTER: [constraints and colouring on the grid (k_solve_grid;
 * 0 when the cluster does them), the cluster kernel (k_solve_cluster)];
 * zeros for a step that ran otherwise. */
int vxp_last_solve_split_ms(vxp_ctx* ctx, float out[2]);

/* Diagnostics: ns from the start of the last step kernel to the end of each
 * of its phases: [start, begin, pairs, cache, probe, finalize, constraints,
 * solve, end, islands, broad phase, sweep setup, sweep substeps, position
 * sweeps, sweep kernel start, broad-phase boxes, broad-phase count pass,
 * broad-phase scan, pair id lookup, pair SAT and regions, sweep slot records,
 * sweep rows] (islands: the IslandManager pass beside the constraint phase;
 * broad phase: the device pair list, when the step builds it; sweep: the
 * shared-memory sweeps of the cluster kernel or a one-CTA world); at most
 * 23 entries.  A phase that did not run this step leaves a stale or zero
 * entry. */
int vxp_phase_times(vxp_ctx* ctx, uint64_t* out, uint32_t n);

/* ---------------------------------------------------------------------------
 * Batched worlds.  No counterpart in the reference (one VoxelPhysicsSystem
 * steps one world); a batch steps many independent worlds at once, each one
 * exactly as vxp_step_device_pairs would, in one kernel launch per step: one
 * CTA per world runs that world's pair source, narrow phase and solver.  The
 * launch is captured once in a CUDA graph and replayed every step.  Worlds
 * share the batch's colliders and configuration; their bodies' collider_id
 * values refer to vxp_batch_collider_upload ids.
 * ------------------------------------------------------------------------- */
typedef struct vxp_batch vxp_batch;

int vxp_batch_create(const vxp_config* cfg, int device, uint32_t max_worlds, vxp_batch** out);
void vxp_batch_destroy(vxp_batch* b);
int vxp_batch_last_error(const vxp_batch* b, char* buf, size_t n);
int vxp_batch_collider_upload(vxp_batch* b, uint32_t collider_id, float voxel_size, const vxp_brick* bricks,
                              uint32_t n_bricks);
/* vxp_collider_edit / vxp_collider_read on the batch's shared colliders (every
 * world whose bodies use the collider sees the edit), and
 * vxp_invalidate_cache_for_body on one world's cache. */
int vxp_batch_collider_edit(vxp_batch* b, uint32_t collider_id, const int32_t* coords,
                            const uint8_t* values, uint32_t n, int mode);
int vxp_batch_collider_read(vxp_batch* b, uint32_t collider_id, vxp_collider_info* info,
                            vxp_brick* bricks, uint32_t cap, uint32_t* n_bricks);
int vxp_batch_invalidate_cache_for_body(vxp_batch* b, uint32_t world, uint32_t body_id,
                                        uint32_t* n_invalidated);
/* (Re)starts world slot `world` with these bodies: empty contact manager and
 * brick-pair cache.  pair_capacity 0 = 16 x n (grown on demand).  A slot
 * that held a world before reuses its device buffers (zeroed, grown when too
 * small): no allocation, and the same results as a new slot. */
int vxp_batch_world_set(vxp_batch* b, uint32_t world, const vxp_body* bodies, uint32_t n, uint32_t pair_capacity);
/* Empties the slot; its device memory stays with it for the next world set
 * there (vxp_batch_world_release frees it). */
int vxp_batch_world_clear(vxp_batch* b, uint32_t world);
/* Empties the slot and frees its device memory (which waits for the device). */
int vxp_batch_world_release(vxp_batch* b, uint32_t world);
int vxp_batch_world_get(vxp_batch* b, uint32_t world, vxp_body* bodies, uint32_t n);
/* vxp_bodies_export for one world of a batch, on the batch's stream. */
int vxp_batch_world_export(vxp_batch* b, uint32_t world, const vxp_state_view* dst, uint32_t first, uint32_t n,
                           int device_memory, void* consumer_stream);
int vxp_batch_world_stats(vxp_batch* b, uint32_t world, vxp_stats* out);
/* Device bytes held by a world slot, occupied or cleared (admission
 * accounting). */
uint64_t vxp_batch_world_bytes(vxp_batch* b, uint32_t world);
/* Every occupied slot advances n_steps steps of dt (queued, not waited for). */
int vxp_batch_step(vxp_batch* b, float dt, uint32_t n_steps);
/* Waits; reports device errors (VXP_ERR_CAP: a world's pair list overflowed
 * and that world left its step undone; its buffers are grown) and grows the
 * pair buffers of worlds close to capacity. */
int vxp_batch_synchronize(vxp_batch* b);
/* Device ms of the last vxp_batch_step call, and per slot the ms of its CTA
 * in the last step (0 for empty slots). */
int vxp_batch_times(vxp_batch* b, float* total_ms, float* world_ms, uint32_t n);
/* Schedule: CTA size 256 or 512; launch order 0 = slot order, 1 = longest
 * measured world first. */
int vxp_batch_set_schedule(vxp_batch* b, uint32_t threads, uint32_t order_mode);
/* Per-world tiles: worlds of at least min_bodies_512 bodies step as
 * 512-thread CTAs, the others as 256-thread CTAs; the two launches run side
 * by side (one graph, two streams).  order_mode as above, within each group.
 * No counterpart in the reference (it steps one world). */
int vxp_batch_set_tiles(vxp_batch* b, uint32_t min_bodies_512, uint32_t order_mode);
/* Autotuner: runs trial_steps real steps under each schedule, keeps the
 * fastest; ms_out[VXP_BATCH_SCHEDULES] = mean step ms of (256,0), (256,1),
 * (512,0), (512,1), then per-world tiles with the 512-thread threshold at
 * 128, 256, 512 and 1024 bodies (longest first).  *choice: the index kept. */
#define VXP_BATCH_SCHEDULES 8
int vxp_batch_autotune(vxp_batch* b, float dt, uint32_t trial_steps, float* ms_out, uint32_t* choice);

/* ---------------------------------------------------------------------------
 * Allocation-free pair source.  No counterpart in the reference (its broad
 * phase is a host AABB tree); this is a variant of the device pair source
 * behind vxp_pairs_from_bodies for callers that cannot let the library
 * allocate device memory: an engine that runs its physics on a frame thread
 * where cudaMalloc's implicit device synchronisation is not allowed, or one
 * whose device memory is all handed out by its own allocator.  It creates no
 * context and calls no cudaMalloc / cudaFree or other allocating routine.
 *
 * All pointers are device memory owned by the caller, for n bodies:
 *   positions, rotations   n x 4 floats (x, y, z, unused) / (x, y, z, w)
 *   local_aabbs            n x 8 floats: min x, y, z, unused, max x, y, z,
 *                          unused; min > max marks a body without collider
 *   ids                    n body ids, strictly ascending (otherwise
 *                          *count is 0 and no pair is written; with
 *                          VXP_CHECK_ARGS=1 in the environment the call
 *                          waits for its work and returns VXP_ERR_ARG)
 *   body_types             n VXP_BODY_* values
 *   out                    room for cap pairs; *count (device) receives the
 *                          total, which may exceed cap (the list is cut)
 * The result equals vxp_pairs_from_bodies for the same bodies and margin.
 * Work is queued on `stream` (a cudaStream_t, or NULL) and is not waited for.
 *
 * Its scratch is one static device array sized for 16384 bodies (about
 * 640 KiB), held by every GPU that loads the library until the process
 * exits; n > 16384 returns VXP_ERR_CAP.  The first call on a device looks up
 * the array's device address (once, with that device current); make that
 * first call before capturing any stream.  Every call uses the same array:
 * calls whose work overlaps on the GPU (other streams, other host threads)
 * race and must be serialised by the caller.  No scratch value carries over
 * from one call to the next.  The device address is kept for the life of
 * the process: do not reset the device while the library is loaded.  An
 * error already pending on the calling thread is left in place and the call
 * returns VXP_ERR_CUDA without launching.
 * ------------------------------------------------------------------------- */
int vxp_pairs_noalloc(const float* positions, const float* rotations, const float* local_aabbs,
                      const uint32_t* ids, const uint32_t* body_types, uint32_t n, float margin,
                      vxp_pair* out, uint32_t cap, uint32_t* count, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* VXP_H */
