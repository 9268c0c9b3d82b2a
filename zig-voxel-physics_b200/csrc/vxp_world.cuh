// vxp_world.cuh — device data layout of one simulated world and the phases of
// one VoxelPhysicsSystem.step (src/system.zig:537-555) on the GPU.
//
// One world is stepped by a "group": either one CTA (BlockGroup; many small
// worlds run side by side, one per CTA) or a whole cooperative grid
// (GridGroup; one large world).  Each phase below is written once against the
// group interface: rank()/size() for thread-parallel loops, warp_id()/nwarps()
// for warp-parallel loops, sync() between phases.  GridGroup.sync() is a
// bounded grid barrier that reports VXP_ERR_TIMEOUT instead of spinning
// forever.
//
// Phase map (reference file:line → phase)
//   system.narrowPhase filter        system.zig:586-655      phase_pairs
//   NarrowPhase.processPair head     narrow_phase.zig:1414-1469 phase_pairs
//   BrickPairCache.get/put           narrow_phase.zig:228-302 cache_replay (in phase_probe)
//   detectVoxelCollisions            narrow_phase.zig:722-857 phase_probe
//   ContactManifold.addContact       narrow_phase.zig:451-481 phase_probe (replay)
//   ContactManager.addManifold       narrow_phase.zig:1011-1059 phase_finalize
//   system.solve / ContactSolver     solver.zig:449-958      phase_constraints..phase_store
//   updateSleepStates                system.zig:786-792      phase_store
#pragma once

#include <cstdint>

#include "vxp_math.cuh"

namespace vxp {

// ---------------------------------------------------------------------------
// Layouts
// ---------------------------------------------------------------------------

// A collider on the device: the reference's hash map of bricks becomes a dense
// brick-coordinate grid of slots into one voxel pool.
struct DCollider {
    float vs;
    int32_t min_bound[3], max_bound[3];   // voxel coords, max exclusive
    float aabb_min[3], aabb_max[3];       // local AABB (recomputeMetadata)
    int32_t bmin[3];                      // brick grid origin
    int32_t bdim[3];                      // brick grid extent
    uint32_t grid_off;                    // into the slot grid
    uint32_t brick_off;                   // first brick in the voxel pool
    uint32_t n_bricks;
    uint32_t solid_count;
    // Neighbourhood masks (kNoTable: none): for every probe centre c in
    // [min_bound - 1, max_bound] per axis (x fastest), a uint4 of 27-bit masks
    // over the centre's 3 x 3 x 3 neighbours inside [min_bound, max_bound)
    // (bit dz*9 + dy*3 + dx, offsets from -1): non-empty, corner, corner or
    // edge, inside.  Built from the voxels when the collider reaches the
    // device, and again after each edit of its voxels.
    uint32_t nb_off;
    // The table's range in the pool: nb_cap entries from nb_base (nb_cap 0:
    // none).  An edit that leaves more probe centres than nb_cap sets nb_off
    // to kNoTable, and the probes fall back to their 27 lookups.
    uint32_t nb_base, nb_cap;
};
constexpr uint32_t kNoTable = 0xFFFFFFFFu;

// Solver / narrow-phase state of one body (BodyState, solver.zig:203-229).
struct __align__(16) DBody {
    float4 p;             // position, w = inv_mass
    float4 q;             // rotation
    float4 v;             // linear velocity
    float4 w;             // angular velocity
    float4 i0, i1, i2;    // world inverse inertia rows (w unused)
};

// Per-body properties that the step reads (BodyProperties, body.zig:103-174)
// and the sleep fields it updates.
struct DBodyProp {
    float il[9];          // inverse inertia, local
    float friction, restitution, lin_damp, ang_damp;
    float sleep_timer;
    uint32_t id, type, collider, sleeping;
};

// Flags of a pair after phase_pairs.
enum : uint32_t {
    PF_INVALID = 1u << 0,   // a body id not found
    PF_CARRY = 1u << 1,     // both sleeping: previous manifold carried over
    PF_DROPPED = 1u << 2,   // beyond the reference's 512-pair cap
    PF_NOCOLL = 1u << 3,    // a body without collider
    PF_SEPARATED = 1u << 4, // SAT early-out
    PF_CACHE = 1u << 5,     // brick-pair cache consulted
    PF_DETECT = 1u << 7,    // detectVoxelCollisions runs
    PF_REGION = 1u << 8,    // overlap region non-empty
    PF_TESTED = 1u << 9,    // processPair was called
    PF_HEAVY = 1u << 10,    // overlap region large enough to be probed by a whole CTA
};

struct PairInfo {
    uint32_t ia, ib;
    uint32_t flags;
    uint32_t hit;           // brick-pair cache: 0 not consulted, 1 hit, 2 miss
    uint32_t cache_slot;    // hit: entry read; miss: entry written
    int32_t rmin[3], rmax[3];
    uint32_t voxels_checked;
    uint32_t candidates;
    uint32_t key_a, key_b;
    unsigned long long th; // transform hash of the cache key
};

// Brick-pair cache entry (BrickPairCacheEntry, narrow_phase.zig:172-177); the
// brick positions of every key the reference builds are (0,0,0).
struct CacheKeyRec {
    uint32_t a, b;
    unsigned long long th;
    unsigned long long last_used;
    uint32_t valid, _pad;
};
struct ContactRec {          // same field order as vxp_contact
    float point[3], normal[3], penetration, la[3], lb[3];
    float normal_impulse, tangent_impulse[2], normal_mass, tangent_mass[2];
    uint32_t _pad;
    unsigned long long feature_id;
};
struct ManifoldRec {         // same layout as vxp_manifold
    uint32_t a, b, n;
    float friction, restitution;
    uint32_t _pad;
    ContactRec c[4];
};
struct CacheValRec {
    ContactRec c[4];
    uint32_t n, has_collision, voxels_checked, _pad;
};

struct HashSlot {            // pairKey -> manifold index
    unsigned long long key;  // 0 = empty (pair keys are never 0: ids > 0)
    uint32_t idx, _pad;
};

// The brick-pair cache table while one warp replays this step's lookups:
// shared-memory arrays of cache_cap entries (key ids, transform hash,
// last-used frame with 0 = empty slot).
constexpr uint32_t kMaxCacheSmem = 4096;
struct CacheSmem {
    uint2* ab;
    unsigned long long* th;
    uint32_t* lu;
};

// Step configuration (vxp_config distilled).
struct StepCfg {
    float gravity[3];
    float dt;
    uint32_t substeps, vel_iters, pos_iters;
    uint32_t disable_rotation;
    float hertz, damping_ratio, pos_rate, max_pos_corr, slop;
    uint32_t warm_starting;
    float warm_scale;
    uint32_t friction_on, restitution_on;
    uint32_t sleeping_on, warm_store_on;
    uint32_t use_sat, use_cache;
    uint32_t reference_caps;
    uint32_t colouring;
    uint32_t dump_candidates;
    uint32_t phases;          // PH_* bits
    uint32_t solver_div;      // grid launch: solver blocks = manifolds / solver_div
    uint32_t device_pairs;    // 1: the step builds its own pair list (phase_broadphase)
    float margin;             // AABB inflation of that pair list
    uint32_t solver_flow;     // 1: sweeps ordered by per-body event counters, 0: colour barriers
    uint32_t flow_smem_chunks;  // constraint chunks per block the launch's shared memory holds
    uint32_t record_substeps;   // 1: write every body's state after each substep to subrec
    uint32_t heavy_voxels;      // overlap regions of at least this many voxels are probed by a CTA (0: never)
    uint32_t count_bricks;      // count the bricks each probed pair touches (C_BRICKS; traffic accounting only)
    uint32_t owner_groups;      // > 1: pack each colour by owner group (home body mod this; the sweep cluster's size)
    uint32_t islands_on;        // IslandManager statistics each solve (PhysicsConfig.enable_islands)
    uint32_t block_smem;        // one-CTA launch: dynamic shared memory the sweeps may hold their state in (0: L2)
};
enum : uint32_t { PH_NARROW = 1u, PH_SOLVE = 2u, PH_SKIP_TEST = 4u, PH_STEP = 7u };

// Per-world counters and flags (device).  Indices of WorldDev::ctr.
enum : uint32_t {
    C_PAIRS_IN = 0,
    C_PAIRS_TESTED,
    C_PAIRS_COLLIDING,
    C_VOXELS_CHECKED,
    C_CONTACTS,
    C_SKIPPED_SLEEPING,
    C_PRESERVED,
    C_CACHE_HITS,
    C_CACHE_MISSES,
    C_CACHE_EVICTIONS,
    C_MANIFOLDS,
    C_CONSTRAINTS,
    C_POINTS,
    C_COLOURS,
    C_POS_ITERS,
    C_STEP_SKIPPED,
    C_MAX_PEN_KEY,   // ordered-int key of max penetration
    C_CANDIDATES,
    C_WORK,          // work counter of phase_probe
    C_DUMP_N,        // candidates dumped
    C_AWAKE,         // dynamic awake bodies seen by the sleep check
    C_BRICKS,        // bricks of A in the overlap region + bricks of B in B's
    C_NCACHE,        // pairs that consult the brick-pair cache this step
    C_KIN_CONTACT,   // constraints touching an awake kinematic body
    C_SOLVE_GO,      // set by the narrow part of a step when its solve part may run
    C_SUBREC,        // substeps recorded in subrec by the last solve
    C_NHEAVY,        // pairs in the CTA-probed list (w.cons during the probe)
    C_HWORK,         // work counter over that list
    C_CONS_M,        // constraint manifolds of the step (solve part split in two kernels)
    C_CONS_NCOL,     // their colours
    C_SWEEP,         // how the cluster sweeps ran (SWEEP_*)
    C_ISL_DIFF,      // the frame's contact graph differs from the last island build's
    C_ISLANDS,       // IslandManager stats of this step: islands,
    C_ISL_SLEEPING,  // sleeping islands,
    C_ISL_LARGEST,   // bodies in the largest island
    C_ERROR = 47,    // sticky error bits (not cleared per step)
    C_NCTR = 48
};
// Phase boundaries recorded in WorldDev::ts by rank 0 (diagnostics).
enum : uint32_t {
    TS_START, TS_BEGIN, TS_PAIRS, TS_CACHE, TS_PROBE, TS_FINALIZE, TS_CONSTRAINTS, TS_SOLVE, TS_END, TS_ISLANDS,
    TS_BROAD, TS_SW_SETUP, TS_SW_SUBSTEPS, TS_SW_POSITION, TS_SW_START,
    // inside the broad phase, the pair filter and the sweep setup
    TS_BP_AABB, TS_BP_COUNT, TS_BP_SCAN, TS_PR_IDS, TS_PR_SAT, TS_SW_SLOTS, TS_SW_ROWS, TS_N = 24
};
// C_SWEEP: the cluster kernel's sweeps with every constraint row in shared
// memory, with the rows that did not fit in global memory, or with all
// state in L2 (colour barriers); 0 when no cluster kernel ran.
enum : uint32_t { SWEEP_SHARED = 1u, SWEEP_SPILL = 2u, SWEEP_L2 = 3u };
static_assert(C_ISL_LARGEST < C_ERROR, "every counter below C_ERROR is cleared each step");
// Island flags (WorldDev::isl_flag) and kept state words (WorldDev::isl_state).
enum : uint32_t { ISL_TOUCHED = 1u, ISL_MOVING = 2u, ISL_ASLEEP = 4u };
enum : uint32_t { IS_DIRTY, IS_TOTAL, IS_LARGEST, IS_NKEYS, IS_BUF, IS_BUILDS, IS_SKIPS, IS_N = 8 };
enum : uint32_t { ERR_TIMEOUT = 1u, ERR_CAP = 2u, ERR_COLOURS = 4u, ERR_OVERFLOW = 8u, ERR_BOUNDS = 16u };

// A brick-pair cache lookup of the step: the pair, its key and the start of
// its probe window (hash % capacity).
struct CacheLook {
    uint32_t p, a, b, start;
    unsigned long long th;
};

struct WorldDev {
    StepCfg cfg;
    uint32_t n_bodies;
    uint32_t n_pairs;             // set from *n_pairs_dev at kernel start
    uint32_t* n_pairs_dev;        // pair count of this step (device)
    uint32_t pair_cap;
    uint32_t ht_cap;              // power of two >= 2 * pair_cap
    uint32_t cache_cap;
    uint32_t dump_cap;
    // bodies
    DBody* body;
    DBodyProp* prop;
    float4* p0;                   // position at step start (writeBack NaN reset)
    float4* qn;                   // normalised rotation per body (transformPoint)
    uint2* ids;                   // (id, index) sorted by id
    // pair source
    float4* aabb_mn;              // inflated world AABB per body (the step's broad phase: in id order)
    float4* aabb_mx;
    uint32_t* pcount;             // pairs per id-sorted row
    uint32_t* bpmask;             // broad-phase hit masks: row s, 32 columns from s + 1 + 32 j at s * bp_stride + j
    uint32_t bp_stride, bp_rows;  // words per row; rows it holds (0: no masks, the sweep runs twice)
    uint32_t* poff;               // their exclusive prefix
    // pairs
    uint2* pairs;                 // (body_a id, body_b id)
    PairInfo* pinfo;
    // contact manager: two manifold arrays / hash tables, flipped per frame
    ManifoldRec* man[2];
    HashSlot* ht[2];
    uint32_t* frame;              // [0] = frame counter (man[frame & 1] is the latest),
                                  // [1] = pair count of the latest manifold array
    // brick-pair cache
    CacheKeyRec* ckey;
    CacheValRec* cval;
    uint32_t* cwriter;            // last pair writing each slot this frame
    CacheLook* clist;             // lookups of the pairs consulting the cache, in pair order
    unsigned long long* cframe;   // cache frame counter
    // constraints
    uint32_t* cons;               // constraint -> pair index (pair order)
    uint32_t* colour;             // per constraint (constraint order)
    uint32_t* pos_of;             // constraint -> packed position (colour-major)
    uint32_t* packed_pair;        // packed position -> pair index
    uint32_t* adj_off;            // body -> adjacency offset (n_bodies + 1)
    uint32_t* adj;                // constraint ids, 2 per constraint at most
    uint32_t* adj_cur;            // fill cursors (n_bodies)
    uint32_t* colour_cnt;         // 257: counts, then offsets
    uint32_t* colour_cur;         // 256 cursors
    uint32_t* ocnt;               // 256 x owner_groups + 1: counts, then offsets of (colour, owner) groups; points at kOwnerPoints
    uint32_t* ocur;               // 256 x owner_groups cursors
    const uint32_t* stat_idx;     // the static bodies, ascending
    uint32_t n_static;
    uint32_t* bmask;              // reference colouring: 8 words per body
    // event-ordered sweeps: per packed manifold (rank on body a, degree of a,
    // rank on body b, degree of b), ~0u for a body the solver never writes;
    // per body the number of sweep events applied so far; per body the state
    // that prepare reads (after gravity), two substeps deep
    uint4* rk;
    uint32_t* ev;
    DBody* snap;
    uint2* chunk;                 // [first, end) positions of <= 32 manifolds of one colour
    float* subrec;                // per substep and body: position, rotation, v, w (13 floats)
    // packed constraint data, slot-major [slot][M]; see CP_* field ids
    float* cp;                    // CP_NFIELDS * 4 * pair_cap floats
    // islands (IslandManager): per body the union-find parent (the island's
    // root, its smallest body index, after a build), ISL_* flags and, per
    // root, its size and sleep timer; the pair keys of the manifolds of two
    // builds (the last one in isl_keys[state[IS_BUF]]); IS_* words kept
    // across steps
    uint32_t* isl_parent;
    uint32_t* isl_flag;
    uint32_t* isl_size;
    float* isl_timer;
    unsigned long long* isl_keys[2];
    uint32_t* isl_state;
    float* crow;                  // CP_NVEL * 4 * pair_cap floats or null: the cluster sweeps'
                                  // point rows that do not fit in shared memory
    uint4* cm;                    // per packed manifold: ia, ib, n, pair
    float2* cfr;                  // per packed manifold: friction, restitution
    // scratch
    uint32_t* scan;               // per-block partials for group scans
    uint32_t* flag;               // per-pair scratch flags (n_pairs)
    uint32_t* ctr;                // C_NCTR counters
    unsigned long long* ts;       // phase timestamps (ns), TS_* slots
    // debug dump
    struct Cand {
        uint32_t pair_index;
        int32_t a[3], b[3];
        uint32_t passed;
        float dist_sq;
    } * dump;
};

// Owner groups the packing can sort each colour into (the largest sweep
// cluster).
constexpr uint32_t kMaxOwnerGroups = 16;
// After the (colour, owner) offsets in ocnt: the points each sweep CTA holds
// by owner (kMaxOwnerGroups), then dealt round-robin (kMaxOwnerGroups).
constexpr uint32_t kOwnerPoints = 256u * kMaxOwnerGroups + 1u;

// Packed constraint-point fields (ConstraintPoint, solver.zig:122-168).  The
// first CP_NVEL are the ones the velocity-type sweeps (warm start, velocity,
// relax) read or write besides tangent2, which is normal x tangent1
// (prepareConstraints); prepare and the position sweeps also read the rest,
// which do not change during the solve.
enum : uint32_t {
    CP_NX, CP_NY, CP_NZ,            // normal
    CP_PX, CP_PY, CP_PZ,            // point
    CP_RAX, CP_RAY, CP_RAZ,         // r_a
    CP_RBX, CP_RBY, CP_RBZ,         // r_b
    CP_T1X, CP_T1Y, CP_T1Z,         // tangent1
    CP_NM, CP_TM0, CP_TM1,          // effective masses
    CP_BIAS,                        // velocity bias
    CP_NI, CP_TI0, CP_TI1,          // accumulated impulses
    CP_NVEL,
    CP_T2X = CP_NVEL, CP_T2Y, CP_T2Z,  // tangent2
    CP_LAX, CP_LAY, CP_LAZ,            // local anchor a
    CP_LBX, CP_LBY, CP_LBZ,            // local anchor b
    CP_BASE,                           // base separation
    CP_NFIELDS
};

}  // namespace vxp
