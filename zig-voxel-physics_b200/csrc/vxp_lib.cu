// vxp_lib.cu — C ABI of the B200 voxel contact + TGS-soft solver library.
//
// Host side: context and device-memory management, collider upload, the pair
// source, kernel launches.  Device side: the step kernels over the phases of
// vxp_step.cuh.  Built with
//   nvcc -gencode arch=compute_100a,code=sm_100a --fmad=false
//        -prec-div=true -prec-sqrt=true -ftz=false
// so that every float operation rounds like the reference's strict f32 code.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/vxp.h"
#include "vxp_math.cuh"
#include "vxp_collider.cuh"
#include "vxp_step.cuh"
#include "vxp_world.cuh"

using namespace vxp;

// ===========================================================================
// Kernels
// ===========================================================================

// Dynamic shared memory: one WarpManifold per warp, then the cache table.
__device__ __forceinline__ CacheSmem cache_smem(unsigned char* raw, uint32_t nwarps, uint32_t cap) {
    unsigned char* p = raw + sizeof(WarpManifold) * nwarps;
    CacheSmem c;
    c.ab = reinterpret_cast<uint2*>(p);
    c.th = reinterpret_cast<unsigned long long*>(p + sizeof(uint2) * cap);
    c.lu = reinterpret_cast<uint32_t*>(p + (sizeof(uint2) + sizeof(unsigned long long)) * cap);
    return c;
}

// One world per CTA: block b steps worlds[b].
template <int kThreads>
__global__ void __launch_bounds__(kThreads, 512 / kThreads) k_step_block(WorldDev* worlds, ColliderSet cs) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    WarpManifold* wsm = reinterpret_cast<WarpManifold*>(smem_raw);
    WorldDev w = worlds[blockIdx.x];
    const CacheSmem csm = cache_smem(smem_raw, blockDim.x / 32u, w.cache_cap);
    BlockGroup g;
    world_step(g, w, cs, wsm, csm, reinterpret_cast<float*>(smem_raw));
}
template __global__ void k_step_block<256>(WorldDev*, ColliderSet);
template __global__ void k_step_block<512>(WorldDev*, ColliderSet);

// One world over a cooperative grid, in two kernels: the narrow part of the
// step, then its solve part (barrier words bar[0] and bar[1]).
__global__ void __launch_bounds__(512, 1) k_step_grid(const WorldDev* world, ColliderSet cs, GridBar* bar,
                                                      unsigned long long timeout_ns) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    WarpManifold* wsm = reinterpret_cast<WarpManifold*>(smem_raw);
    WorldDev w = *world;
    const CacheSmem csm = cache_smem(smem_raw, blockDim.x / 32u, w.cache_cap);
    GridGroup g{bar, &w.ctr[C_ERROR], timeout_ns, gridDim.x};
    world_step_narrow(g, w, cs, wsm, csm);
}
__global__ void __launch_bounds__(256, 1) k_solve_grid(const WorldDev* world, GridBar* bar,
                                                       unsigned long long timeout_ns, uint32_t part) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    WorldDev w = *world;
    GridGroup g{bar, &w.ctr[C_ERROR], timeout_ns, gridDim.x};
    world_step_solve(g, w, reinterpret_cast<float*>(smem_raw), true, part);
}
// The solve part on one thread-block cluster (the whole grid): all of it
// (whole) or the sweeps and the store after k_solve_grid(...,
// SOLVE_CONSTRAINTS).
__global__ void __launch_bounds__(256, 1) k_solve_cluster(const WorldDev* world, uint32_t smem_bytes, uint32_t whole) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint32_t ncta;
    asm("mov.u32 %0, %%cluster_nctarank;" : "=r"(ncta));
    WorldDev w = *world;
    if (ncta != gridDim.x) {  // launch constants: the same verdict in every block
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(&w.ctr[C_ERROR], ERR_BOUNDS);
        return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && w.ts) w.ts[TS_SW_START] = global_ns();
    ClusterGroup g;
    world_step_sweeps(g, w, smem_raw, smem_bytes, whole != 0u);
}

// Pair source: world AABB of each body's collider (AABB.transform,
// math.zig:686-693) inflated by margin.
// VoxelBody.getWorldAABB (body.zig:430-435): the collider's local AABB
// through AABB.transform (math.zig:686-693), or the position for a body
// without a collider.
__device__ __forceinline__ void body_world_aabb(const DBody& b, const DBodyProp& pr, const ColliderSet& cs, F3& lo,
                                                F3& hi) {
    const F3 x = f3of(b.p);
    const Qt q = qof(b.q);
    if (pr.collider < cs.n) {
        const DCollider& c = cs.c[pr.collider];
        const float inf = __int_as_float(0x7f800000);
        lo = F3{inf, inf, inf};
        hi = F3{-inf, -inf, -inf};
        for (int k = 0; k < 8; ++k) {
            const F3 corner{(k & 1) ? c.aabb_max[0] : c.aabb_min[0], (k & 2) ? c.aabb_max[1] : c.aabb_min[1],
                            (k & 4) ? c.aabb_max[2] : c.aabb_min[2]};
            const F3 p = transform_point(x, q, corner);
            lo = min3(lo, p);
            hi = max3(hi, p);
        }
    } else {
        lo = x;
        hi = x;
    }
}

__global__ void k_body_aabbs(const DBody* body, const DBodyProp* prop, uint32_t n, ColliderSet cs, float margin,
                             float4* mn, float4* mx) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    F3 lo, hi;
    body_world_aabb(body[i], prop[i], cs, lo, hi);
    lo = lo - F3{margin, margin, margin};
    hi = hi + F3{margin, margin, margin};
    mn[i] = make_float4(lo.x, lo.y, lo.z, 0.f);
    mx[i] = make_float4(hi.x, hi.y, hi.z, 0.f);
}

// The body table as vxp_body records (vxp_bodies_get): one thread a body,
// packed on the device so that the host reads it back in one copy.
__global__ void k_pack_bodies(const DBody* body, const DBodyProp* prop, const uint32_t* pub_cid, uint32_t n,
                              vxp_body* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const DBody d = body[i];
    const DBodyProp& p = prop[i];
    vxp_body s;
    s.id = p.id;
    s.body_type = p.type;
    s.collider_id = pub_cid[i];
    s.is_sleeping = p.sleeping;
    s.position[0] = d.p.x; s.position[1] = d.p.y; s.position[2] = d.p.z;
    s.rotation[0] = d.q.x; s.rotation[1] = d.q.y; s.rotation[2] = d.q.z; s.rotation[3] = d.q.w;
    s.linear_velocity[0] = d.v.x; s.linear_velocity[1] = d.v.y; s.linear_velocity[2] = d.v.z;
    s.angular_velocity[0] = d.w.x; s.angular_velocity[1] = d.w.y; s.angular_velocity[2] = d.w.z;
    s.inv_mass = d.p.w;
    for (int k = 0; k < 9; ++k) s.inv_inertia_local[k] = p.il[k];
    s.friction = p.friction;
    s.restitution = p.restitution;
    s.linear_damping = p.lin_damp;
    s.angular_damping = p.ang_damp;
    s.sleep_timer = p.sleep_timer;
    out[i] = s;
}

// Bulk state export of bodies [first, first + n): one thread a body, each
// requested field into its own array (vxp_bodies_export).
__global__ void k_export(const DBody* body, const DBodyProp* prop, uint32_t first, uint32_t n, ColliderSet cs,
                         vxp_state_view d) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const uint32_t i = first + j;
    const DBody b = body[i];
    if (d.position) {
        d.position[3u * j] = b.p.x;
        d.position[3u * j + 1u] = b.p.y;
        d.position[3u * j + 2u] = b.p.z;
    }
    if (d.rotation) {  // scalar stores: the caller's array need only be 4-byte aligned
        d.rotation[4u * j] = b.q.x;
        d.rotation[4u * j + 1u] = b.q.y;
        d.rotation[4u * j + 2u] = b.q.z;
        d.rotation[4u * j + 3u] = b.q.w;
    }
    if (d.linear_velocity) {
        d.linear_velocity[3u * j] = b.v.x;
        d.linear_velocity[3u * j + 1u] = b.v.y;
        d.linear_velocity[3u * j + 2u] = b.v.z;
    }
    if (d.angular_velocity) {
        d.angular_velocity[3u * j] = b.w.x;
        d.angular_velocity[3u * j + 1u] = b.w.y;
        d.angular_velocity[3u * j + 2u] = b.w.z;
    }
    if (d.aabb_min || d.aabb_max) {
        F3 lo, hi;
        body_world_aabb(b, prop[i], cs, lo, hi);
        if (d.aabb_min) {
            d.aabb_min[3u * j] = lo.x;
            d.aabb_min[3u * j + 1u] = lo.y;
            d.aabb_min[3u * j + 2u] = lo.z;
        }
        if (d.aabb_max) {
            d.aabb_max[3u * j] = hi.x;
            d.aabb_max[3u * j + 1u] = hi.y;
            d.aabb_max[3u * j + 2u] = hi.z;
        }
    }
    if (d.sleeping) d.sleeping[j] = prop[i].sleeping ? 1u : 0u;
}

// Pairs (s < t in id order) whose inflated AABBs overlap and that are not
// both static.  One warp per row s; lanes sweep t in strides of 32 and a
// ballot keeps the row's pairs in t order.  Pass 0 counts per row, pass 1
// writes at the scanned offsets (clamped to cap).
// masks (row stride mstride words, or null): the count pass keeps each row's
// 32-column hit masks there and the write pass reads them instead of testing
// the boxes again.
__global__ void k_pairs(const uint2* ids, const DBodyProp* prop, uint32_t n, const float4* mn, const float4* mx,
                        uint32_t* counts, const uint32_t* offsets, uint2* out, uint32_t cap, int pass,
                        uint32_t* masks, uint32_t mstride) {
    const uint32_t s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31;
    if (s >= n) return;
    const uint2 is = ids[s];
    if (pass && masks) {
        const uint32_t nj = (n - 1u - s + 31u) / 32u;
        const uint32_t* mrow = masks + (size_t)s * mstride;
        uint32_t o = offsets[s];
        for (uint32_t jb = 0; jb < nj; jb += 32u) {
            const uint32_t j = jb + lane;
            uint32_t mk = j < nj ? mrow[j] : 0u;
            const uint32_t c = (uint32_t)__popc(mk);
            const uint32_t inc = warp_incl_scan(c);
            uint32_t q = o + inc - c;
            for (; mk; mk &= mk - 1u, ++q)
                if (q < cap) out[q] = make_uint2(is.x, ids[s + 1u + 32u * j + (uint32_t)(__ffs(mk) - 1)].x);
            o += __shfl_sync(0xffffffffu, inc, 31);
        }
        return;
    }
    const float4 a0 = mn[is.y], a1 = mx[is.y];
    const bool si = prop[is.y].type == 0u;
    uint32_t o = pass ? offsets[s] : 0u;
    uint32_t cnt = 0;
    for (uint32_t t0 = s + 1; t0 < n; t0 += 32u) {
        const uint32_t t = t0 + lane;
        bool hit = false;
        uint2 it = make_uint2(0u, 0u);
        if (t < n) {
            it = ids[t];
            if (!(si && prop[it.y].type == 0u)) {
                const float4 b0 = mn[it.y], b1 = mx[it.y];
                hit = a0.x <= b1.x && a1.x >= b0.x && a0.y <= b1.y && a1.y >= b0.y && a0.z <= b1.z && a1.z >= b0.z;
            }
        }
        const uint32_t m = __ballot_sync(0xffffffffu, hit);
        if (masks && lane == 0) masks[(size_t)s * mstride + (t0 - s - 1u) / 32u] = m;
        if (pass && hit) {
            const uint32_t slot = o + __popc(m & ((1u << lane) - 1u));
            if (slot < cap) out[slot] = make_uint2(is.x, it.x);
        }
        o += __popc(m);
        cnt += __popc(m);
    }
    if (!pass && lane == 0) counts[s] = cnt;
}

// Exclusive scan of counts (single block, n arbitrary); writes total to *total.
__global__ void __launch_bounds__(1024) k_scan1(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* total) {
    uint32_t carry = 0;
    for (uint32_t t0 = 0; t0 < n; t0 += blockDim.x) {
        const uint32_t i = t0 + threadIdx.x;
        const uint32_t v = i < n ? in[i] : 0u;
        uint32_t tile;
        const uint32_t ex = block_excl_scan(v, &tile);
        if (i < n) out[i] = carry + ex;
        carry += tile;
    }
    if (threadIdx.x == 0) *total = carry;
}

// Rebuild a manifold hash table after the manifold buffers were re-allocated.
__global__ void k_rehash(const ManifoldRec* man, uint32_t n, HashSlot* ht, uint32_t cap) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    if (man[p].n > 0u) ht_insert(ht, cap, pair_key(man[p].a, man[p].b), p);
}

// ===========================================================================
// Host side
// ===========================================================================
namespace {

template <class T> struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    ~DBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    cudaError_t reserve(size_t k, bool keep = false) {
        if (k <= n && p) return cudaSuccess;
        T* q = nullptr;
        const size_t bytes = std::max<size_t>(k, 1) * sizeof(T);
        cudaError_t e = cudaMalloc(&q, bytes);
        if (e != cudaSuccess) return e;
        cudaMemset(q, 0, bytes);
        if (keep && p && n) cudaMemcpy(q, p, n * sizeof(T), cudaMemcpyDeviceToDevice);
        if (p) cudaFree(p);
        p = q;
        n = std::max<size_t>(k, 1);
        return cudaSuccess;
    }
    size_t bytes() const { return n * sizeof(T); }
};

uint32_t next_pow2(uint32_t x) {
    uint32_t p = 1;
    while (p < x) p <<= 1;
    return p;
}

std::string fmt(const char* f, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, f);
    vsnprintf(buf, sizeof(buf), f, ap);
    va_end(ap);
    return buf;
}

constexpr uint32_t kBlockThreads = 512;
// CTA sizes of the two cooperative grid kernels of a large world's step (one
// CTA per SM each): the narrow part wants many warps to hide its memory
// latency, the solve part wants registers for its long dependent chains.
constexpr uint32_t kGridThreads = 512;
constexpr uint32_t kSolveThreads = 256;
size_t step_smem(uint32_t threads, uint32_t cache_cap) {
    return sizeof(WarpManifold) * (threads / 32) +
           (size_t)cache_cap * (sizeof(uint2) + sizeof(unsigned long long) + sizeof(uint32_t));
}
// The grid solve kernel (one CTA per SM) keeps up to kGridFlowChunks chunks
// of constraint rows per block in shared memory.
constexpr uint32_t kGridFlowChunks = 4;
size_t grid_smem(uint32_t cache_cap) { return step_smem(kGridThreads, cache_cap); }
// Dynamic shared memory of a one-CTA world's launch (either CTA size): the
// narrow part's warp scratch and cache table, then room for the sweeps' state
// of a small world (bodies, manifold slots, point rows); two 256-thread CTAs
// still fit on one SM.
constexpr size_t kBlockSolveSmem = 96 * 1024;
size_t block_smem(uint32_t cache_cap) { return std::max(step_smem(512, cache_cap), kBlockSolveSmem); }
size_t solve_smem() { return (size_t)kGridFlowChunks * kChunkFloats * sizeof(float); }
uint32_t flow_chunks(size_t smem) { return (uint32_t)(smem / (kChunkFloats * sizeof(float))); }

uint64_t hash_brick_pos(int32_t x, int32_t y, int32_t z) {  // collider.zig:187-192
    const uint64_t ux = (uint64_t)(int64_t)x, uy = (uint64_t)(int64_t)y, uz = (uint64_t)(int64_t)z;
    return ux ^ (uy * 0x517cc1b727220a95ull) ^ (uz * 0x9e3779b97f4a7c15ull);
}

// VoxelCollider.recomputeMetadata (collider.zig:283-333), bricks in the order
// given: bounds over the solid voxels (max exclusive; zero when none is
// solid), the local AABB as the merge of the bricks' solid-voxel boxes, the
// solid count.
struct ColliderMeta {
    int32_t min_bound[3], max_bound[3];
    float aabb_min[3], aabb_max[3];
    uint32_t solid;
};
void collider_metadata(float vs, const int32_t* pos, const uint8_t* vox, size_t nb, ColliderMeta& h) {
    h.solid = 0;
    for (int k = 0; k < 3; ++k) {
        h.min_bound[k] = INT32_MAX;
        h.max_bound[k] = INT32_MIN;
    }
    const float inf = __builtin_inff();
    float amn[3] = {inf, inf, inf}, amx[3] = {-inf, -inf, -inf};
    for (size_t b = 0; b < nb; ++b) {
        const int32_t* bp = &pos[b * 3];
        const uint8_t* v = &vox[b * 512];
        uint32_t solid = 0;
        float bmn[3] = {inf, inf, inf}, bmx[3] = {-inf, -inf, -inf};
        for (int i = 0; i < 512; ++i) {
            if ((v[i] & 7u) == 0u) continue;
            ++solid;
            const int c[3] = {i % 8, (i / 8) % 8, i / 64};
            for (int k = 0; k < 3; ++k) {
                const float lp = ((float)bp[k] * 8.0f + (float)c[k]) * vs;
                bmn[k] = std::fmin(bmn[k], lp);
                bmx[k] = std::fmax(bmx[k], lp + vs);
                const int32_t vc = bp[k] * 8 + c[k];
                h.min_bound[k] = std::min(h.min_bound[k], vc);
                h.max_bound[k] = std::max(h.max_bound[k], vc + 1);
            }
        }
        if (solid == 0) continue;
        h.solid += solid;
        for (int k = 0; k < 3; ++k) {
            amn[k] = std::fmin(amn[k], bmn[k]);
            amx[k] = std::fmax(amx[k], bmx[k]);
        }
    }
    if (h.solid == 0)
        for (int k = 0; k < 3; ++k) h.min_bound[k] = h.max_bound[k] = 0;
    for (int k = 0; k < 3; ++k) {
        h.aabb_min[k] = amn[k];
        h.aabb_max[k] = amx[k];
    }
}

// Floor division by the brick size (voxelToBrickPos, collider.zig:195-201).
inline int32_t brick_of(int32_t v) { return v >= 0 ? v / 8 : -((-v + 7) / 8); }

struct VoxelKey {
    int32_t x, y, z;
    bool operator==(const VoxelKey& o) const { return x == o.x && y == o.y && z == o.z; }
};
struct VoxelKeyHash {
    size_t operator()(const VoxelKey& k) const {
        return (size_t)(((uint64_t)(uint32_t)k.x * 0x9E3779B97F4A7C15ull) ^
                        ((uint64_t)(uint32_t)k.y * 0xC2B2AE3D27D4EB4Full) ^ ((uint64_t)(uint32_t)k.z << 1));
    }
};

// The colliders of a context or batch on the device.  Per collider: a dense
// grid of brick slots (each cell resolved by hashBrickPos, as the reference's
// brick map resolves it) over the box of its bricks plus one brick on every
// side, its bricks' voxels and positions in two pools, and a neighbourhood-mask
// table.  The pools grow by appending: an upload places only its own collider,
// an edit runs in place on the device, and an edit that needs new bricks
// places its collider again from a copy of its voxels.  Ranges left behind by
// replaced placements are reclaimed by a full re-placement once they outweigh
// the live ones.
struct ColliderStore {
    struct Entry {
        uint32_t id = 0;
        float vs = 0.0f;
        std::vector<int32_t> pos;                        // 3 per brick, the device's brick order
        std::unordered_map<uint64_t, uint32_t> by_hash;  // hashBrickPos -> brick
        std::vector<int32_t> cover;                      // further brick cells the grid covers (3 each)
        std::vector<uint8_t> staged;                     // voxels waiting for placement (512 per brick)
        bool placed = false;
        bool aliased = false;    // some grid cell reaches a brick of another position (shared hash)
        DCollider d{};           // the layout as placed; the metadata then lives on the device
        size_t grid_cells = 0;
    };
    std::vector<Entry> colliders;
    std::unordered_map<uint32_t, uint32_t> index;
    DBuf<DCollider> d_col;
    DBuf<int32_t> d_grid;
    DBuf<uint8_t> d_vox;
    DBuf<int4> d_bpos;
    DBuf<uint4> d_nb;
    DBuf<uint32_t> d_list;
    DBuf<EditScratch> d_scratch;
    size_t grid_used = 0, brick_used = 0, nb_used = 0;
    size_t grid_dead = 0, brick_dead = 0, nb_dead = 0;
    uint32_t n_dev = 0;
    bool dirty = false;    // colliders wait for placement
    bool replace = false;  // every collider is placed again (tables switched)
    // neighbourhood-mask tables: colliders with at most kNbMaxCentres probe
    // centres get one, while the pool stays within kNbMaxTotal entries (16 B
    // each: 4 GiB at most, e.g. 2.4 GB for 512 colliders of 64^3 voxels)
    static constexpr uint64_t kNbMaxCentres = 1ull << 23, kNbMaxTotal = 1ull << 28;
    static constexpr size_t kMaxGridCells = (size_t)1 << 28;
    bool tables = true;  // build neighbourhood-mask tables at all
    // pinned staging of edit lists, two in turn, each free again once the
    // kernels of the edit that used it have run
    struct Staging {
        int4* host = nullptr;
        size_t cap = 0;
        DBuf<int4> dev;
        cudaEvent_t done = nullptr;
    };
    Staging stage[2];
    uint32_t turn = 0;

    ColliderStore() = default;
    ColliderStore(const ColliderStore&) = delete;
    ColliderStore& operator=(const ColliderStore&) = delete;
    ~ColliderStore() {
        for (Staging& s : stage) {
            if (s.done) cudaEventDestroy(s.done);
            if (s.host) cudaFreeHost(s.host);
        }
    }

    int upload(uint32_t id, float vs, const vxp_brick* bricks, uint32_t n, std::string& err) {
        if (!bricks && n) {
            err = "null bricks";
            return VXP_ERR_ARG;
        }
        if (!(vs > 0.0f)) {
            err = "voxel_size must be positive";
            return VXP_ERR_ARG;
        }
        Entry e;
        e.id = id;
        e.vs = vs;
        e.pos.resize((size_t)n * 3);
        e.staged.resize((size_t)n * 512);
        for (uint32_t i = 0; i < n; ++i) {
            for (int k = 0; k < 3; ++k) e.pos[(size_t)i * 3 + k] = bricks[i].pos[k];
            std::memcpy(&e.staged[(size_t)i * 512], bricks[i].voxels, 512);
            const uint64_t hb = hash_brick_pos(bricks[i].pos[0], bricks[i].pos[1], bricks[i].pos[2]);
            auto ins = e.by_hash.emplace(hb, i);
            if (!ins.second) {
                err = fmt("collider %u: bricks %u and %u share a hashBrickPos value", id, ins.first->second, i);
                return VXP_ERR_ARG;
            }
        }
        auto it = index.find(id);
        if (it != index.end()) {
            retire(colliders[it->second]);
            colliders[it->second] = std::move(e);
        } else {
            index[id] = (uint32_t)colliders.size();
            colliders.push_back(std::move(e));
        }
        dirty = true;
        return VXP_OK;
    }
    uint32_t index_of(uint32_t id) const {
        auto it = index.find(id);
        return it == index.end() ? 0xFFFFFFFFu : it->second;
    }
    void set_tables(bool on) {
        if (tables == on) return;
        tables = on;
        replace = dirty = true;
    }
    ColliderSet set() const { return ColliderSet{d_col.p, d_grid.p, d_vox.p, n_dev, d_nb.p}; }

    // Places every collider that waits, on `s` (ordered after the work
    // already there), and reclaims dead ranges when they outweigh the live.
    int sync(cudaStream_t s, std::string& err) {
        if (!d_col.p && (d_col.reserve(1) != cudaSuccess || d_grid.reserve(1) != cudaSuccess ||
                         d_vox.reserve(512) != cudaSuccess || d_bpos.reserve(1) != cudaSuccess ||
                         d_nb.reserve(1) != cudaSuccess)) {
            err = "collider store: device allocation failed";
            return VXP_ERR_OOM;
        }
        if (!dirty) return VXP_OK;
        const bool reclaim = (brick_dead > 4096 && brick_dead > brick_used - brick_dead) ||
                             (nb_dead > ((size_t)1 << 20) && nb_dead > nb_used - nb_dead) ||
                             (grid_dead > ((size_t)1 << 20) && grid_dead > grid_used - grid_dead);
        if (replace || reclaim) {
            if (int rc = fetch_all(s, err)) return rc;
            grid_used = brick_used = nb_used = 0;
            grid_dead = brick_dead = nb_dead = 0;
            for (Entry& e : colliders) e.placed = false;
            replace = false;
        }
        std::vector<uint32_t> todo;
        for (uint32_t i = 0; i < colliders.size(); ++i)
            if (!colliders[i].placed) todo.push_back(i);
        if (int rc = place(todo, s, err)) return rc;
        dirty = false;
        return VXP_OK;
    }

    // The current metadata and bricks of collider `id`, read from the device.
    int read(uint32_t id, vxp_collider_info* info, vxp_brick* bricks, uint32_t cap, uint32_t* n_out,
             cudaStream_t s, std::string& err) {
        const uint32_t ci = index_of(id);
        if (ci == 0xFFFFFFFFu) {
            err = fmt("collider %u was never uploaded", id);
            return VXP_ERR_ARG;
        }
        if (int rc = sync(s, err)) return rc;
        if (cudaStreamSynchronize(s) != cudaSuccess) {
            err = "collider read: stream failed";
            return VXP_ERR_CUDA;
        }
        const Entry& e = colliders[ci];
        DCollider d;
        if (cudaMemcpy(&d, d_col.p + ci, sizeof(d), cudaMemcpyDeviceToHost) != cudaSuccess) {
            err = "collider read: copy failed";
            return VXP_ERR_CUDA;
        }
        const uint32_t n = d.n_bricks;
        if (info) {
            std::memset(info, 0, sizeof(*info));
            info->voxel_size = d.vs;
            for (int k = 0; k < 3; ++k) {
                info->min_bound[k] = d.min_bound[k];
                info->max_bound[k] = d.max_bound[k];
                info->aabb_min[k] = d.aabb_min[k];
                info->aabb_max[k] = d.aabb_max[k];
            }
            info->solid_count = d.solid_count;
            info->n_bricks = n;
            info->has_table = d.nb_off != kNoTable ? 1u : 0u;
        }
        if (n_out) *n_out = n;
        const uint32_t k = bricks ? std::min(cap, n) : 0u;
        if (k) {
            std::vector<uint8_t> v((size_t)k * 512);
            if (cudaMemcpy(v.data(), d_vox.p + (size_t)d.brick_off * 512, v.size(), cudaMemcpyDeviceToHost) !=
                cudaSuccess) {
                err = "collider read: copy failed";
                return VXP_ERR_CUDA;
            }
            for (uint32_t b = 0; b < k; ++b) {
                for (int q = 0; q < 3; ++q) bricks[b].pos[q] = e.pos[(size_t)b * 3 + q];
                std::memcpy(bricks[b].voxels, &v[(size_t)b * 512], 512);
            }
        }
        return VXP_OK;
    }

    // An edit batch of collider `id` (vxp_collider_edit), queued on `s`.
    int edit(uint32_t id, const int32_t* coords, const uint8_t* values, uint32_t n, uint32_t mode, cudaStream_t s,
             std::string& err) {
        const uint32_t ci = index_of(id);
        if (ci == 0xFFFFFFFFu) {
            err = fmt("collider %u was never uploaded", id);
            return VXP_ERR_ARG;
        }
        if ((n && (!coords || !values)) || mode > EDIT_OCCUPANCY || n > (1u << 24)) {
            err = "collider edit: bad arguments";
            return VXP_ERR_ARG;
        }
        if (n == 0) return VXP_OK;
        if (int rc = sync(s, err)) return rc;
        Entry& e = colliders[ci];
        // one entry per voxel, the last write winning; new bricks in the
        // order the writes first reach them (getOrCreateBrick)
        std::vector<int4> list;
        list.reserve(n);
        std::unordered_map<VoxelKey, uint32_t, VoxelKeyHash> seen;
        seen.reserve((size_t)n * 2);
        std::vector<int32_t> fresh;                   // new brick positions, 3 each
        std::unordered_map<uint64_t, bool> fresh_at;  // by hash
        std::vector<int32_t> extra;                   // held cells whose neighbours leave the grid
        for (uint32_t i = 0; i < n; ++i) {
            const int32_t x = coords[(size_t)i * 3], y = coords[(size_t)i * 3 + 1], z = coords[(size_t)i * 3 + 2];
            const int32_t w = mode == EDIT_SET ? (int32_t)values[i] : (values[i] ? 1 : 0);
            auto ins = seen.emplace(VoxelKey{x, y, z}, (uint32_t)list.size());
            if (!ins.second) {
                list[ins.first->second].w = w;
                continue;
            }
            list.push_back(make_int4(x, y, z, w));
            const int32_t bx = brick_of(x), by = brick_of(y), bz = brick_of(z);
            const uint64_t hb = hash_brick_pos(bx, by, bz);
            if (!e.by_hash.count(hb)) {
                if (fresh_at.emplace(hb, true).second) {
                    fresh.push_back(bx);
                    fresh.push_back(by);
                    fresh.push_back(bz);
                }
            } else if (!in_grid(e.d, bx - 1, by - 1, bz - 1) || !in_grid(e.d, bx + 1, by + 1, bz + 1)) {
                extra.push_back(bx);
                extra.push_back(by);
                extra.push_back(bz);
            }
        }
        if (!fresh.empty() || !extra.empty()) {
            // place the collider again with the new bricks (zeroed) and a grid
            // that covers every cell the edit reads or writes
            if (int rc = fetch(ci, s, err)) return rc;
            const size_t nb0 = e.pos.size() / 3;
            for (size_t b = 0; b < fresh.size() / 3; ++b) {
                e.by_hash.emplace(hash_brick_pos(fresh[b * 3], fresh[b * 3 + 1], fresh[b * 3 + 2]),
                                  (uint32_t)(nb0 + b));
                e.pos.insert(e.pos.end(), &fresh[b * 3], &fresh[b * 3] + 3);
            }
            e.staged.resize(e.pos.size() / 3 * 512, 0);
            e.cover.insert(e.cover.end(), extra.begin(), extra.end());
            retire(e);
            std::vector<uint32_t> one{ci};
            if (int rc = place(one, s, err)) return rc;
        }
        // Where one brick serves several cells of the grid (a shared
        // hashBrickPos), distinct coordinates can reach one voxel byte: each
        // such byte then takes the last value the list writes to it, and one
        // re-typing, the last in the reference's order (list order, then the
        // voxel before its -x, +x, -y, +y, -z, +z neighbours); and any table
        // entry may read a changed byte, so the whole table is rebuilt.
        std::vector<int4> targets;
        const bool shared = e.aliased;
        if (shared) {
            auto byte_of = [&](int32_t x, int32_t y, int32_t z, uint64_t* key) {
                auto it = e.by_hash.find(hash_brick_pos(brick_of(x), brick_of(y), brick_of(z)));
                if (it == e.by_hash.end()) return false;
                *key = ((uint64_t)it->second << 9) | (uint64_t)((x & 7) + 8 * (y & 7) + 64 * (z & 7));
                return true;
            };
            std::unordered_map<uint64_t, int32_t> last;
            uint64_t key = 0;
            for (uint32_t i = 0; i < n; ++i)
                if (byte_of(coords[(size_t)i * 3], coords[(size_t)i * 3 + 1], coords[(size_t)i * 3 + 2], &key))
                    last[key] = mode == EDIT_SET ? (int32_t)values[i] : (values[i] ? 1 : 0);
            for (int4& q : list)
                if (byte_of(q.x, q.y, q.z, &key)) q.w = last[key];
            if (mode == EDIT_OCCUPANCY) {
                const int32_t off[7][3] = {{0, 0, 0}, {-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
                std::unordered_map<uint64_t, uint32_t> who;
                for (uint32_t i = 0; i < n; ++i)
                    for (int k = 0; k < 7; ++k) {
                        const int32_t x = coords[(size_t)i * 3] + off[k][0], y = coords[(size_t)i * 3 + 1] + off[k][1],
                                      z = coords[(size_t)i * 3 + 2] + off[k][2];
                        if (!byte_of(x, y, z, &key)) continue;
                        auto r = who.emplace(key, (uint32_t)targets.size());
                        if (r.second) targets.push_back(make_int4(x, y, z, 0));
                        else targets[r.first->second] = make_int4(x, y, z, 0);
                    }
            }
        }
        // the lists through pinned staging: the writes, then the re-typings
        const size_t total = list.size() + targets.size();
        Staging& st = stage[turn];
        turn ^= 1u;
        if (st.done && cudaEventSynchronize(st.done) != cudaSuccess) {
            err = "collider edit: stream failed";
            return VXP_ERR_CUDA;
        }
        if (!st.done && cudaEventCreateWithFlags(&st.done, cudaEventDisableTiming) != cudaSuccess) {
            err = "collider edit: event";
            return VXP_ERR_CUDA;
        }
        if (st.cap < total) {
            if (st.host) cudaFreeHost(st.host);
            st.host = nullptr;
            st.cap = 0;
            const size_t want = std::max<size_t>(total, 1024);
            if (cudaMallocHost(&st.host, want * sizeof(int4)) != cudaSuccess || st.dev.reserve(want) != cudaSuccess) {
                err = "collider edit: allocation failed";
                return VXP_ERR_OOM;
            }
            st.cap = want;
        }
        if (d_scratch.reserve(1) != cudaSuccess) {
            err = "collider edit: allocation failed";
            return VXP_ERR_OOM;
        }
        std::memcpy(st.host, list.data(), list.size() * sizeof(int4));
        if (!targets.empty()) std::memcpy(st.host + list.size(), targets.data(), targets.size() * sizeof(int4));
        if (cudaMemcpyAsync(st.dev.p, st.host, total * sizeof(int4), cudaMemcpyHostToDevice, s) != cudaSuccess) {
            err = "collider edit: copy failed";
            return VXP_ERR_CUDA;
        }
        const uint32_t m = (uint32_t)list.size(), t = (uint32_t)targets.size();
        const uint32_t tb = 256;
        k_edit_apply<<<(m + tb - 1) / tb, tb, 0, s>>>(d_col.p, ci, d_grid.p, d_vox.p, st.dev.p, m, mode);
        if (mode == EDIT_OCCUPANCY && !shared)
            k_edit_classify<<<(m * 7u + tb - 1) / tb, tb, 0, s>>>(d_col.p, ci, d_grid.p, d_vox.p, st.dev.p, m, 7u);
        else if (mode == EDIT_OCCUPANCY && t)
            k_edit_classify<<<(t + tb - 1) / tb, tb, 0, s>>>(d_col.p, ci, d_grid.p, d_vox.p, st.dev.p + m, t, 1u);
        const uint32_t nb = e.d.n_bricks;
        const uint32_t mb = std::max<uint32_t>(1u, std::min<uint32_t>(kMetaBlocks, (nb * 32u + kMetaThreads - 1) /
                                                                                       kMetaThreads));
        k_edit_meta<<<mb, kMetaThreads, 0, s>>>(d_col.p, ci, d_vox.p, d_bpos.p, d_scratch.p, shared ? 1u : 0u);
        if (e.d.nb_cap) {
            if (!shared)
                k_edit_table_local<<<(m * 125u + tb - 1) / tb, tb, 0, s>>>(set(), d_nb.p, ci, st.dev.p, m,
                                                                           d_scratch.p);
            const uint32_t fb = std::min<uint32_t>(148u * 4u, (e.d.nb_cap + tb - 1) / tb);
            k_edit_table_full<<<fb, tb, 0, s>>>(set(), d_nb.p, ci, d_scratch.p);
        }
        const cudaError_t le = cudaGetLastError();
        if (le != cudaSuccess || cudaEventRecord(st.done, s) != cudaSuccess) {
            err = fmt("collider edit: launch failed: %s", cudaGetErrorString(le));
            return VXP_ERR_CUDA;
        }
        return VXP_OK;
    }

  private:
    static bool in_grid(const DCollider& d, int32_t bx, int32_t by, int32_t bz) {
        return (uint32_t)(bx - d.bmin[0]) < (uint32_t)d.bdim[0] && (uint32_t)(by - d.bmin[1]) < (uint32_t)d.bdim[1] &&
               (uint32_t)(bz - d.bmin[2]) < (uint32_t)d.bdim[2];
    }
    // A placement's ranges become dead.
    void retire(Entry& e) {
        if (!e.placed) return;
        grid_dead += e.grid_cells;
        brick_dead += e.d.n_bricks;
        nb_dead += e.d.nb_cap;
        e.placed = false;
        dirty = true;
    }
    // Collider ci's voxels as the device holds them, into its staging copy.
    int fetch(uint32_t ci, cudaStream_t s, std::string& err) {
        Entry& e = colliders[ci];
        if (!e.placed) return VXP_OK;
        e.staged.resize((size_t)e.d.n_bricks * 512);
        if (cudaStreamSynchronize(s) != cudaSuccess ||
            (!e.staged.empty() && cudaMemcpy(e.staged.data(), d_vox.p + (size_t)e.d.brick_off * 512,
                                             e.staged.size(), cudaMemcpyDeviceToHost) != cudaSuccess)) {
            err = "collider store: read-back failed";
            return VXP_ERR_CUDA;
        }
        return VXP_OK;
    }
    int fetch_all(cudaStream_t s, std::string& err) {
        if (cudaStreamSynchronize(s) != cudaSuccess) {
            err = "collider store: stream failed";
            return VXP_ERR_CUDA;
        }
        std::vector<uint8_t> all(brick_used * 512);
        if (!all.empty() && cudaMemcpy(all.data(), d_vox.p, all.size(), cudaMemcpyDeviceToHost) != cudaSuccess) {
            err = "collider store: read-back failed";
            return VXP_ERR_CUDA;
        }
        for (Entry& e : colliders) {
            if (!e.placed) continue;
            const size_t off = (size_t)e.d.brick_off * 512;
            e.staged.assign(all.begin() + (ptrdiff_t)off, all.begin() + (ptrdiff_t)(off + (size_t)e.d.n_bricks * 512));
        }
        return VXP_OK;
    }
    // Appends the listed colliders (from their staging copies) to the pools,
    // writes their records and builds their tables.
    int place(const std::vector<uint32_t>& todo, cudaStream_t s, std::string& err) {
        if (todo.empty()) return VXP_OK;
        std::vector<int32_t> grid;
        std::vector<uint8_t> vox;
        std::vector<int4> bpos;
        std::vector<uint32_t> built;
        const size_t g0 = grid_used, b0 = brick_used;
        for (uint32_t ci : todo) {
            Entry& e = colliders[ci];
            const size_t nb = e.pos.size() / 3;
            ColliderMeta h;
            collider_metadata(e.vs, e.pos.data(), e.staged.data(), nb, h);
            DCollider& d = e.d;
            std::memset(&d, 0, sizeof(d));
            d.vs = e.vs;
            for (int k = 0; k < 3; ++k) {
                d.min_bound[k] = h.min_bound[k];
                d.max_bound[k] = h.max_bound[k];
                d.aabb_min[k] = h.aabb_min[k];
                d.aabb_max[k] = h.aabb_max[k];
            }
            d.solid_count = h.solid;
            // grid: the box of the bricks and the extra cells, one brick wider
            // on every side; a collider without bricks gets one empty cell
            int32_t lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
            bool any = false;
            auto grow = [&](const int32_t* p) {
                for (int k = 0; k < 3; ++k) {
                    lo[k] = any ? std::min(lo[k], p[k] - 1) : p[k] - 1;
                    hi[k] = any ? std::max(hi[k], p[k] + 1) : p[k] + 1;
                }
                any = true;
            };
            for (size_t b = 0; b < nb; ++b) grow(&e.pos[b * 3]);
            for (size_t c = 0; c < e.cover.size() / 3; ++c) grow(&e.cover[c * 3]);
            size_t cells = 1;
            for (int k = 0; k < 3; ++k) {
                d.bmin[k] = lo[k];
                d.bdim[k] = hi[k] - lo[k] + 1;
                cells *= (size_t)d.bdim[k];
            }
            if (cells > kMaxGridCells) {
                err = fmt("collider %u brick grid too large", e.id);
                return VXP_ERR_CAP;
            }
            d.grid_off = (uint32_t)(g0 + grid.size());
            d.brick_off = (uint32_t)(b0 + bpos.size());
            d.n_bricks = (uint32_t)nb;
            const size_t gbase = grid.size();
            grid.resize(gbase + cells, -1);
            bool aliased = false;
            for (int32_t bz = lo[2]; bz <= hi[2]; ++bz)
                for (int32_t by = lo[1]; by <= hi[1]; ++by)
                    for (int32_t bx = lo[0]; bx <= hi[0]; ++bx) {
                        auto it = e.by_hash.find(hash_brick_pos(bx, by, bz));
                        if (it == e.by_hash.end()) continue;
                        const int32_t* own = &e.pos[(size_t)it->second * 3];
                        aliased |= own[0] != bx || own[1] != by || own[2] != bz;
                        grid[gbase + (size_t)(bx - lo[0]) +
                             (size_t)d.bdim[0] * ((size_t)(by - lo[1]) + (size_t)d.bdim[1] * (size_t)(bz - lo[2]))] =
                            (int32_t)it->second;
                    }
            e.grid_cells = cells;
            e.aliased = aliased;
            vox.insert(vox.end(), e.staged.begin(), e.staged.end());
            for (size_t b = 0; b < nb; ++b) bpos.push_back(make_int4(e.pos[b * 3], e.pos[b * 3 + 1], e.pos[b * 3 + 2], 0));
            uint64_t centres = 1;
            for (int k = 0; k < 3; ++k) centres *= (uint64_t)((int64_t)h.max_bound[k] - h.min_bound[k] + 2);
            if (tables && centres <= kNbMaxCentres && nb_used + centres <= kNbMaxTotal) {
                d.nb_base = d.nb_off = (uint32_t)nb_used;
                d.nb_cap = (uint32_t)centres;
                nb_used += centres;
                built.push_back(ci);
            } else {
                d.nb_off = kNoTable;
                d.nb_base = d.nb_cap = 0;
            }
        }
        const size_t ng = g0 + grid.size(), nbk = b0 + bpos.size();
        // growing a pool copies it and frees the old one: nothing may still read it
        if (cudaStreamSynchronize(s) != cudaSuccess) {
            err = "collider store: stream failed";
            return VXP_ERR_CUDA;
        }
        auto room = [](size_t need, size_t have) { return need <= have ? have : std::max(need, 2 * have); };
        if (d_col.reserve(room(colliders.size(), d_col.p ? d_col.n : 0), true) != cudaSuccess ||
            d_grid.reserve(room(ng, d_grid.p ? d_grid.n : 0), true) != cudaSuccess ||
            d_vox.reserve(room(nbk * 512, d_vox.p ? d_vox.n : 0), true) != cudaSuccess ||
            d_bpos.reserve(room(nbk, d_bpos.p ? d_bpos.n : 0), true) != cudaSuccess ||
            (nb_used && d_nb.reserve(room(nb_used, d_nb.p ? d_nb.n : 0), true) != cudaSuccess) ||
            (!built.empty() && d_list.reserve(built.size()) != cudaSuccess)) {
            err = "collider upload: device allocation failed";
            return VXP_ERR_OOM;
        }
        bool ok = (grid.empty() || cudaMemcpy(d_grid.p + g0, grid.data(), grid.size() * sizeof(int32_t),
                                              cudaMemcpyHostToDevice) == cudaSuccess) &&
                  (vox.empty() || cudaMemcpy(d_vox.p + b0 * 512, vox.data(), vox.size(), cudaMemcpyHostToDevice) ==
                                      cudaSuccess) &&
                  (bpos.empty() || cudaMemcpy(d_bpos.p + b0, bpos.data(), bpos.size() * sizeof(int4),
                                              cudaMemcpyHostToDevice) == cudaSuccess);
        // records, one copy per run of consecutive indices
        for (size_t i = 0; ok && i < todo.size();) {
            size_t j = i + 1;
            while (j < todo.size() && todo[j] == todo[j - 1] + 1) ++j;
            std::vector<DCollider> run(j - i);
            for (size_t k = i; k < j; ++k) run[k - i] = colliders[todo[k]].d;
            ok = cudaMemcpy(d_col.p + todo[i], run.data(), run.size() * sizeof(DCollider), cudaMemcpyHostToDevice) ==
                 cudaSuccess;
            i = j;
        }
        if (!ok) {
            err = "collider upload: copy failed";
            return VXP_ERR_CUDA;
        }
        grid_used = ng;
        brick_used = nbk;
        n_dev = (uint32_t)colliders.size();
        for (uint32_t ci : todo) {
            Entry& e = colliders[ci];
            e.placed = true;
            std::vector<uint8_t>().swap(e.staged);
        }
        if (!built.empty()) {
            if (cudaMemcpy(d_list.p, built.data(), built.size() * sizeof(uint32_t), cudaMemcpyHostToDevice) !=
                cudaSuccess) {
                err = "collider upload: copy failed";
                return VXP_ERR_CUDA;
            }
            const dim3 grid_dims(64, std::min<uint32_t>((uint32_t)built.size(), 65535u));
            k_nbhd_build<<<grid_dims, 256, 0, s>>>(set(), d_nb.p, d_list.p, (uint32_t)built.size());
            if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) {
                err = "collider upload: neighbourhood tables failed";
                return VXP_ERR_CUDA;
            }
        }
        return VXP_OK;
    }
};

StepCfg step_cfg(const vxp_config& c, float dt, uint32_t dump, uint32_t phases) {
    StepCfg s;
    std::memset(&s, 0, sizeof(s));
    for (int i = 0; i < 3; ++i) s.gravity[i] = c.gravity[i];
    s.dt = dt;
    s.substeps = c.substeps;
    s.vel_iters = c.velocity_iterations;
    s.pos_iters = c.position_iterations;
    s.disable_rotation = c.disable_rotation;
    s.hertz = c.hertz;
    s.damping_ratio = c.damping_ratio;
    s.pos_rate = c.position_correction_rate;
    s.max_pos_corr = c.max_position_correction;
    s.slop = c.slop;
    s.warm_starting = c.warm_starting;
    s.warm_scale = c.warm_start_scale;
    s.friction_on = c.enable_friction;
    s.restitution_on = c.enable_restitution;
    s.sleeping_on = c.enable_sleeping;
    s.warm_store_on = c.enable_warm_starting;
    s.use_sat = c.use_brick_sat;
    s.use_cache = c.use_brick_pair_cache;
    s.reference_caps = c.reference_caps;
    s.colouring = c.colouring;
    s.dump_candidates = dump;
    s.phases = phases;
    s.solver_div = 128;
    s.device_pairs = 0;
    s.margin = 0.1f;
    s.solver_flow = 1;
    s.heavy_voxels = 1024;  // batches of small worlds: one CTA per world
    s.count_bricks = 0;
    s.owner_groups = 1;
    s.islands_on = c.enable_islands;
    return s;
}

// Device memory of one world: body state, pair list, contact manager, cache,
// constraint arrays and scratch.
struct WorldBuffers {
    uint32_t n_bodies = 0, body_cap = 0, pair_cap = 0, ht_cap = 0, cache_cap = 1024, dump_cap = 0, scan_blocks = 1;
    bool live = true;  // a batch slot whose world was cleared keeps its buffers with live = false
    // a context's world (swept by a cluster) keeps a global home for the
    // constraint rows that do not fit in the cluster's shared memory
    bool spill_rows = false;
    std::vector<uint32_t> collider_public;
    DBuf<DBody> body;
    DBuf<DBodyProp> prop;
    DBuf<float4> p0, qn, aabb_mn, aabb_mx;
    DBuf<uint2> ids;
    DBuf<uint32_t> pcount, poff, adj_off, adj_cur, bmask, bpmask;
    uint32_t bp_stride = 0, bp_rows = 0;
    // worlds of at most this many bodies keep the broad phase's hit masks
    // (rows x rows / 32 words) and sweep their AABBs once
    static constexpr uint32_t kMaskBodies = 8192;
    DBuf<uint2> pairs;
    DBuf<uint32_t> n_pairs_dev;
    DBuf<PairInfo> pinfo;
    DBuf<ManifoldRec> man0, man1;
    DBuf<HashSlot> ht0, ht1;
    DBuf<uint32_t> frame;
    DBuf<uint32_t> cons, colour, pos_of, packed_pair, adj, flag;
    DBuf<CacheLook> clist;
    DBuf<float> cp, crow;
    // islands: per body, per pair slot (two builds' keys), kept state words
    DBuf<uint32_t> isl_parent, isl_flag, isl_size, isl_state;
    DBuf<float> isl_timer;
    DBuf<unsigned long long> isl_keys0, isl_keys1;
    DBuf<uint4> cm, rk;
    DBuf<float2> cfr;
    DBuf<uint32_t> ev;
    DBuf<DBody> snap;
    DBuf<uint2> chunk;
    DBuf<uint32_t> colour_cnt, colour_cur, scan, ctr, cwriter, ocnt, ocur, stat;
    uint32_t n_static = 0;
    DBuf<unsigned long long> ts, cframe;
    DBuf<CacheKeyRec> ckey;
    DBuf<CacheValRec> cval;
    DBuf<WorldDev::Cand> dump;
    DBuf<unsigned char> export_stage;  // host-memory exports land here first
    DBuf<uint32_t> pub_cid;            // per body: its collider id as the caller named it
    DBuf<vxp_body> pack;               // vxp_bodies_get's records, packed on the device

    int init(uint32_t cache, uint32_t blocks, std::string& err) {
        cache_cap = cache;
        scan_blocks = blocks;
        bool ok = true;
        ok &= n_pairs_dev.reserve(1) == cudaSuccess;
        ok &= frame.reserve(2) == cudaSuccess;
        ok &= colour_cnt.reserve(257) == cudaSuccess;
        ok &= colour_cur.reserve(256) == cudaSuccess;
        ok &= ocnt.reserve(kOwnerPoints + 2 * kMaxOwnerGroups) == cudaSuccess;
        ok &= ocur.reserve(256 * kMaxOwnerGroups) == cudaSuccess;
        ok &= scan.reserve(blocks + 64) == cudaSuccess;
        ok &= ctr.reserve(C_NCTR) == cudaSuccess;
        ok &= ts.reserve(TS_N) == cudaSuccess;
        ok &= ckey.reserve(cache) == cudaSuccess;
        ok &= cval.reserve(cache) == cudaSuccess;
        ok &= cwriter.reserve(cache) == cudaSuccess;
        ok &= cframe.reserve(1) == cudaSuccess;
        ok &= isl_state.reserve(IS_N + (size_t)blocks) == cudaSuccess;  // + the island pass's scan partials
        if (ok) mark_islands_dirty();
        if (!ok) {
            err = "world buffers: device allocation failed";
            return VXP_ERR_OOM;
        }
        return VXP_OK;
    }

    // Grows every pair-sized buffer to hold `need` pairs; keeps the latest
    // frame's manifolds and rebuilds their hash table.
    int ensure_pairs(uint32_t need, std::string& err) {
        if (need <= pair_cap && pair_cap) return VXP_OK;
        uint32_t cap = std::max<uint32_t>(1024, pair_cap);
        while (cap < need) cap *= 2;
        const uint32_t old_cap = pair_cap;
        const uint32_t new_ht = next_pow2(cap * 2);
        bool ok = true;
        ok &= pairs.reserve(cap) == cudaSuccess;
        ok &= pinfo.reserve(cap) == cudaSuccess;
        ok &= man0.reserve(cap, true) == cudaSuccess;
        ok &= man1.reserve(cap, true) == cudaSuccess;
        ok &= cons.reserve(cap) == cudaSuccess;
        ok &= colour.reserve(cap) == cudaSuccess;
        ok &= pos_of.reserve(cap) == cudaSuccess;
        ok &= packed_pair.reserve(cap) == cudaSuccess;
        ok &= adj.reserve((size_t)2 * cap) == cudaSuccess;
        ok &= flag.reserve(cap) == cudaSuccess;
        ok &= clist.reserve(cap) == cudaSuccess;
        ok &= cp.reserve((size_t)CP_NFIELDS * 4 * cap) == cudaSuccess;
        if (spill_rows) ok &= crow.reserve((size_t)CP_NVEL * 4 * cap) == cudaSuccess;
        ok &= isl_keys0.reserve(cap, true) == cudaSuccess;
        ok &= isl_keys1.reserve(cap, true) == cudaSuccess;
        ok &= cm.reserve(cap) == cudaSuccess;
        ok &= rk.reserve(cap) == cudaSuccess;
        ok &= chunk.reserve((size_t)cap / 32 + 257) == cudaSuccess;
        ok &= cfr.reserve(cap) == cudaSuccess;
        if (!ok) {
            err = fmt("pair buffers: device allocation of %u pairs failed", cap);
            return VXP_ERR_OOM;
        }
        if (new_ht != ht_cap) {
            ht0.release();
            ht1.release();
            if (ht0.reserve(new_ht) != cudaSuccess || ht1.reserve(new_ht) != cudaSuccess) {
                err = "hash tables: allocation failed";
                return VXP_ERR_OOM;
            }
            ht_cap = new_ht;
            if (old_cap) {
                uint32_t fr[2] = {0, 0};
                if (cudaMemcpy(fr, frame.p, sizeof(fr), cudaMemcpyDeviceToHost) != cudaSuccess) {
                    err = "frame read failed";
                    return VXP_ERR_CUDA;
                }
                const uint32_t latest_n = fr[1];
                const uint32_t latest = fr[0] & 1u;  // the next step reads it as previous
                if (latest_n) {
                    ManifoldRec* m = latest ? man1.p : man0.p;
                    HashSlot* h = latest ? ht1.p : ht0.p;
                    k_rehash<<<(latest_n + 255) / 256, 256>>>(m, latest_n, h, new_ht);
                    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) {
                        err = "rehash failed";
                        return VXP_ERR_CUDA;
                    }
                }
            }
        }
        pair_cap = cap;
        return VXP_OK;
    }

    int ensure_bodies(uint32_t n, std::string& err) {
        if (n <= body_cap && body_cap) return VXP_OK;
        uint32_t cap = std::max<uint32_t>(64, body_cap);
        while (cap < n) cap *= 2;
        bool ok = true;
        ok &= body.reserve(cap) == cudaSuccess;
        ok &= prop.reserve(cap) == cudaSuccess;
        ok &= p0.reserve(cap) == cudaSuccess;
        ok &= qn.reserve(cap) == cudaSuccess;
        ok &= aabb_mn.reserve(cap) == cudaSuccess;
        ok &= aabb_mx.reserve(cap) == cudaSuccess;
        ok &= ids.reserve(cap) == cudaSuccess;
        ok &= pcount.reserve(cap) == cudaSuccess;
        ok &= poff.reserve(cap) == cudaSuccess;
        ok &= adj_off.reserve((size_t)cap + 1) == cudaSuccess;
        ok &= adj_cur.reserve(cap) == cudaSuccess;
        ok &= bmask.reserve((size_t)cap * 8) == cudaSuccess;
        if (cap <= kMaskBodies) {
            ok &= bpmask.reserve((size_t)cap * ((cap + 31u) / 32u)) == cudaSuccess;
            bp_stride = (cap + 31u) / 32u;
            bp_rows = cap;
        } else {
            bpmask.release();
            bp_stride = bp_rows = 0;
        }
        ok &= ev.reserve(cap) == cudaSuccess;
        ok &= snap.reserve((size_t)cap * 2) == cudaSuccess;
        ok &= isl_parent.reserve(cap) == cudaSuccess;
        ok &= isl_flag.reserve(cap) == cudaSuccess;
        ok &= isl_size.reserve(cap) == cudaSuccess;
        ok &= isl_timer.reserve(cap) == cudaSuccess;
        if (!ok) {
            err = fmt("body buffers: device allocation of %u bodies failed", cap);
            return VXP_ERR_OOM;
        }
        body_cap = cap;
        return VXP_OK;
    }

    int set_bodies(const vxp_body* b, uint32_t n, const ColliderStore& cols, std::string& err) {
        if (!b && n) {
            err = "null bodies";
            return VXP_ERR_ARG;
        }
        if (int rc = ensure_bodies(n, err)) return rc;
        std::vector<DBody> db(n);
        std::vector<DBodyProp> dp(n);
        std::vector<uint2> id(n);
        collider_public.resize(n);
        for (uint32_t i = 0; i < n; ++i) {
            const vxp_body& s = b[i];
            if (s.body_type > 2u) {
                err = fmt("body %u: bad body_type %u", i, s.body_type);
                return VXP_ERR_ARG;
            }
            DBody& d = db[i];
            d.p = make_float4(s.position[0], s.position[1], s.position[2], s.inv_mass);
            d.q = make_float4(s.rotation[0], s.rotation[1], s.rotation[2], s.rotation[3]);
            d.v = make_float4(s.linear_velocity[0], s.linear_velocity[1], s.linear_velocity[2], 0.f);
            d.w = make_float4(s.angular_velocity[0], s.angular_velocity[1], s.angular_velocity[2], 0.f);
            d.i0 = d.i1 = d.i2 = make_float4(0.f, 0.f, 0.f, 0.f);
            DBodyProp& p = dp[i];
            for (int k = 0; k < 9; ++k) p.il[k] = s.inv_inertia_local[k];
            p.friction = s.friction;
            p.restitution = s.restitution;
            p.lin_damp = s.linear_damping;
            p.ang_damp = s.angular_damping;
            p.sleep_timer = s.sleep_timer;
            p.id = s.id;
            p.type = s.body_type;
            p.collider = cols.index_of(s.collider_id);
            p.sleeping = s.is_sleeping ? 1u : 0u;
            collider_public[i] = s.collider_id;
            id[i] = make_uint2(s.id, i);
        }
        std::sort(id.begin(), id.end(), [](const uint2& x, const uint2& y) { return x.x < y.x; });
        for (uint32_t i = 1; i < n; ++i)
            if (id[i].x == id[i - 1].x) {
                err = fmt("duplicate body id %u", id[i].x);
                return VXP_ERR_ARG;
            }
        if (n && (cudaMemcpy(body.p, db.data(), n * sizeof(DBody), cudaMemcpyHostToDevice) != cudaSuccess ||
                  cudaMemcpy(prop.p, dp.data(), n * sizeof(DBodyProp), cudaMemcpyHostToDevice) != cudaSuccess ||
                  cudaMemcpy(ids.p, id.data(), n * sizeof(uint2), cudaMemcpyHostToDevice) != cudaSuccess ||
                  pub_cid.reserve(n) != cudaSuccess || pack.reserve(n) != cudaSuccess ||
                  cudaMemcpy(pub_cid.p, collider_public.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice) !=
                      cudaSuccess)) {
            err = "body upload failed";
            return VXP_ERR_CUDA;
        }
        // the static bodies (never moved by a step), ascending
        std::vector<uint32_t> st;
        for (uint32_t i = 0; i < n; ++i)
            if (dp[i].type == 0u) st.push_back(i);
        if (stat.reserve(std::max<size_t>(st.size(), 1)) != cudaSuccess ||
            (!st.empty() && cudaMemcpy(stat.p, st.data(), st.size() * sizeof(uint32_t), cudaMemcpyHostToDevice) !=
                                cudaSuccess)) {
            err = "static body list upload failed";
            return VXP_ERR_CUDA;
        }
        n_static = (uint32_t)st.size();
        n_bodies = n;
        mark_islands_dirty();  // the island roots are body indices
        return VXP_OK;
    }

    int get_bodies(vxp_body* b, uint32_t n, cudaStream_t stream, std::string& err) {
        if (n != n_bodies) {
            err = fmt("expected %u bodies, got %u", n_bodies, n);
            return VXP_ERR_ARG;
        }
        if (!n) return VXP_OK;
        k_pack_bodies<<<(n + 255u) / 256u, 256, 0, stream>>>(body.p, prop.p, pub_cid.p, n, pack.p);
        if (cudaPeekAtLastError() != cudaSuccess ||
            cudaMemcpyAsync(b, pack.p, n * sizeof(vxp_body), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
            cudaStreamSynchronize(stream) != cudaSuccess) {
            err = "body download failed";
            return VXP_ERR_CUDA;
        }
        return VXP_OK;
    }

    WorldDev make(const vxp_config& cfg, float dt, uint32_t phases, uint32_t solver_div, bool device_pairs,
                  float margin, uint32_t solver_flow) const {
        WorldDev w;
        std::memset(&w, 0, sizeof(w));
        w.cfg = step_cfg(cfg, dt, dump_cap ? 1u : 0u, phases);
        w.cfg.solver_div = solver_div;
        w.cfg.solver_flow = solver_flow;
        w.cfg.device_pairs = device_pairs ? 1u : 0u;
        w.cfg.margin = margin;
        w.n_bodies = n_bodies;
        w.n_pairs_dev = n_pairs_dev.p;
        w.pair_cap = pair_cap;
        w.ht_cap = ht_cap;
        w.cache_cap = cache_cap;
        w.dump_cap = dump_cap;
        w.body = body.p;
        w.prop = prop.p;
        w.p0 = p0.p;
        w.qn = qn.p;
        w.ids = ids.p;
        w.aabb_mn = aabb_mn.p;
        w.aabb_mx = aabb_mx.p;
        w.pcount = pcount.p;
        w.poff = poff.p;
        w.bpmask = bp_rows ? bpmask.p : nullptr;
        w.bp_stride = bp_stride;
        w.bp_rows = bp_rows;
        w.pairs = pairs.p;
        w.pinfo = pinfo.p;
        w.man[0] = man0.p;
        w.man[1] = man1.p;
        w.ht[0] = ht0.p;
        w.ht[1] = ht1.p;
        w.frame = frame.p;
        w.ckey = ckey.p;
        w.cval = cval.p;
        w.cwriter = cwriter.p;
        w.clist = clist.p;
        w.cframe = cframe.p;
        w.cons = cons.p;
        w.colour = colour.p;
        w.pos_of = pos_of.p;
        w.packed_pair = packed_pair.p;
        w.adj_off = adj_off.p;
        w.adj = adj.p;
        w.adj_cur = adj_cur.p;
        w.colour_cnt = colour_cnt.p;
        w.colour_cur = colour_cur.p;
        w.ocnt = ocnt.p;
        w.ocur = ocur.p;
        w.stat_idx = stat.p;
        w.n_static = n_static;
        w.bmask = bmask.p;
        w.cp = cp.p;
        w.crow = crow.p;
        w.isl_parent = isl_parent.p;
        w.isl_flag = isl_flag.p;
        w.isl_size = isl_size.p;
        w.isl_timer = isl_timer.p;
        w.isl_keys[0] = isl_keys0.p;
        w.isl_keys[1] = isl_keys1.p;
        w.isl_state = isl_state.p;
        w.cm = cm.p;
        w.rk = rk.p;
        w.ev = ev.p;
        w.snap = snap.p;
        w.chunk = chunk.p;
        w.cfr = cfr.p;
        w.scan = scan.p;
        w.flag = flag.p;
        w.ctr = ctr.p;
        w.ts = ts.p;
        w.dump = dump.p;
        return w;
    }

    // Every device buffer back to zero, as a new allocation is: a batch slot
    // reused for another world starts from exactly the state of a new one.
    cudaError_t zero_all(cudaStream_t s) {
        cudaError_t e = cudaSuccess;
        auto z = [&](auto& b) {
            if (b.p && e == cudaSuccess) e = cudaMemsetAsync(b.p, 0, b.bytes(), s);
        };
        z(body); z(prop); z(p0); z(qn); z(aabb_mn); z(aabb_mx); z(ids); z(pcount); z(poff); z(adj_off); z(adj_cur);
        z(bmask); z(pairs); z(n_pairs_dev); z(pinfo); z(man0); z(man1); z(ht0); z(ht1); z(frame); z(cons); z(colour);
        z(pos_of); z(packed_pair); z(adj); z(flag); z(clist); z(cp); z(cm); z(rk); z(cfr); z(ev); z(snap); z(chunk);
        z(colour_cnt); z(colour_cur); z(scan); z(ctr); z(cwriter); z(ts); z(cframe); z(ckey); z(cval); z(dump);
        z(ocnt); z(ocur); z(stat); z(bpmask);
        return e;
    }

    size_t device_bytes() const {
        return body.bytes() + prop.bytes() + p0.bytes() + qn.bytes() + aabb_mn.bytes() + aabb_mx.bytes() +
               ids.bytes() + pcount.bytes() + poff.bytes() + adj_off.bytes() + adj_cur.bytes() + bmask.bytes() +
               pairs.bytes() + pinfo.bytes() + man0.bytes() + man1.bytes() + ht0.bytes() + ht1.bytes() +
               cons.bytes() + colour.bytes() + pos_of.bytes() + packed_pair.bytes() + adj.bytes() + flag.bytes() +
               clist.bytes() + cp.bytes() + cm.bytes() + rk.bytes() + ev.bytes() + snap.bytes() + chunk.bytes() + cfr.bytes() +
               ckey.bytes() + cval.bytes() +
               cwriter.bytes() + scan.bytes() + ctr.bytes() + ts.bytes() + dump.bytes() + ocnt.bytes() + ocur.bytes() +
               stat.bytes() + bpmask.bytes() + crow.bytes() + isl_parent.bytes() + isl_flag.bytes() +
               isl_size.bytes() + isl_timer.bytes() + isl_keys0.bytes() + isl_keys1.bytes() + isl_state.bytes() +
               export_stage.bytes() + pub_cid.bytes() + pack.bytes();
    }

    // The next solve rebuilds its islands (IslandManager.markDirty,
    // islands.zig:301-303): at creation and whenever the bodies are replaced.
    void mark_islands_dirty() {
        const uint32_t st[IS_N] = {1u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
        cudaMemcpy(isl_state.p, st, sizeof(st), cudaMemcpyHostToDevice);
    }

    // Counters -> vxp_stats.
    int stats(vxp_stats* s, uint32_t pairs_in, cudaStream_t stream, std::string& err) const {
        uint32_t c[C_NCTR];
        if (cudaMemcpyAsync(c, ctr.p, sizeof(c), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
            cudaStreamSynchronize(stream) != cudaSuccess) {
            err = "counter read failed";
            return VXP_ERR_CUDA;
        }
        std::memset(s, 0, sizeof(*s));
        s->pairs_in = pairs_in;
        s->pairs_tested = c[C_PAIRS_TESTED];
        s->pairs_colliding = c[C_PAIRS_COLLIDING];
        s->voxels_checked = c[C_VOXELS_CHECKED];
        s->contacts_generated = c[C_CONTACTS];
        s->pairs_skipped_sleeping = c[C_SKIPPED_SLEEPING];
        s->manifolds_preserved = c[C_PRESERVED];
        s->cache_hits = c[C_CACHE_HITS];
        s->cache_misses = c[C_CACHE_MISSES];
        s->cache_evictions = c[C_CACHE_EVICTIONS];
        s->manifolds = c[C_MANIFOLDS];
        s->constraints = c[C_CONSTRAINTS];
        s->contact_points = c[C_POINTS];
        s->colours = c[C_COLOURS];
        s->position_iterations_run = c[C_POS_ITERS];
        s->step_skipped = c[C_STEP_SKIPPED];
        const int32_t k = (int32_t)c[C_MAX_PEN_KEY];
        int32_t bits = k >= 0 ? k : (k ^ 0x7FFFFFFF);
        std::memcpy(&s->max_penetration, &bits, 4);
        s->candidates = c[C_CANDIDATES];
        s->bricks_touched = c[C_BRICKS];
        s->sweep_path = c[C_SWEEP];
        s->island_count = c[C_ISLANDS];
        s->sleeping_islands = c[C_ISL_SLEEPING];
        s->active_islands = c[C_ISLANDS] - c[C_ISL_SLEEPING];
        s->largest_island_size = c[C_ISL_LARGEST];
        return VXP_OK;
    }

    // Reads and clears the sticky error word.
    int take_error(cudaStream_t stream, std::string& err) const {
        uint32_t e = 0;
        if (cudaMemcpyAsync(&e, ctr.p + C_ERROR, sizeof(e), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
            cudaStreamSynchronize(stream) != cudaSuccess) {
            err = "error word read failed";
            return VXP_ERR_CUDA;
        }
        if (!e) return VXP_OK;
        const uint32_t z = 0;
        cudaMemcpy(ctr.p + C_ERROR, &z, sizeof(z), cudaMemcpyHostToDevice);
        if (e & ERR_TIMEOUT) {
            err = fmt("a grid barrier or solver wait ran out (error bits 0x%x)", e);
            return VXP_ERR_TIMEOUT;
        }
        if (e & ERR_BOUNDS) {
            err = fmt("an index of the solver's constraint table was out of range (error bits 0x%x)", e);
            return VXP_ERR_STATE;
        }
        if (e & ERR_CAP) {
            err = fmt("pair list exceeded the device capacity; the step left the state untouched (bits 0x%x)", e);
            return VXP_ERR_CAP;
        }
        if (e & ERR_COLOURS) {
            err = fmt("more than 255 colours needed (error bits 0x%x)", e);
            return VXP_ERR_CAP;
        }
        err = fmt("device error bits 0x%x", e);
        return VXP_ERR_STATE;
    }
};

}  // namespace

struct vxp_ctx {
    vxp_config cfg;
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    int sm_count = 148;
    ColliderStore cols;
    WorldBuffers w;
    DBuf<WorldDev> d_world;
    DBuf<GridBar> bar;
    DBuf<uint32_t> pair_counts, pair_offsets;
    uint32_t grid_blocks = 0;
    uint32_t last_pairs = 0;
    cudaEvent_t ev_start = nullptr, ev0 = nullptr, ev1 = nullptr, ev_count = nullptr, ev_mid = nullptr,
                ev_cons = nullptr;
    uint32_t cluster_size = 0;  // CTAs of the cluster that runs the sweeps (0: no cluster launch here)
    uint32_t cluster_smem = 0;  // dynamic shared memory of each of its CTAs
    uint32_t cluster_state_cap = 0xFFFFFFFFu;  // of which the sweeps' state may use at most this
    bool cluster_whole = false;  // the cluster also builds the constraint table and colours it
    bool last_cluster = false;
    bool last_grid = false;
    uint32_t* h_count = nullptr;  // pinned mirror of the device pair count
    bool count_pending = false;
    int use_grid = -1;  // -1 auto, 0 block, 1 grid
    uint32_t solver_div = 128;
    uint32_t solver_flow = 1;
    uint32_t heavy_voxels = 2048;
    unsigned long long wait_limit_ns = 0;  // grid-barrier wait limit; 0: kGridWaitNs
    bool count_bricks = false;  // traffic accounting (C_BRICKS)
    bool record_substeps = false;
    DBuf<float> subrec;
    DBuf<uint32_t> d_word;  // a count read back by the host
};

namespace {

int fail(vxp_ctx* c, int code, const char* f, ...) {
    if (c) {
        char buf[512];
        va_list ap;
        va_start(ap, f);
        vsnprintf(buf, sizeof(buf), f, ap);
        va_end(ap);
        c->err = buf;
    }
    return code;
}
#define CK(call)                                                                                         \
    do {                                                                                                 \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess) return fail(ctx, VXP_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

// Launch configuration of k_solve_cluster: one cluster of n CTAs with smem
// bytes of dynamic shared memory each.
static void cluster_config(cudaLaunchConfig_t* lc, cudaLaunchAttribute* at, uint32_t n, uint32_t smem,
                           cudaStream_t stream) {
    lc->gridDim = dim3(n);
    lc->blockDim = dim3(kSolveThreads);
    lc->dynamicSmemBytes = smem;
    lc->stream = stream;
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = n;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    lc->attrs = at;
    lc->numAttrs = 1;
}

// Longest wait of a block at a grid barrier before it gives up (ERR_TIMEOUT).
constexpr unsigned long long kGridWaitNs = 10ull * 1000ull * 1000ull * 1000ull;

// Runs the step kernel.  device_pairs: the kernel builds the pair list itself.
int launch_step(vxp_ctx* ctx, float dt, uint32_t phases, bool device_pairs, float margin) {
    if (int rc = ctx->cols.sync(ctx->stream, ctx->err)) return rc;
    const bool grid = ctx->use_grid == 1 || (ctx->use_grid < 0 && ctx->w.n_bodies >= 512);
    const bool cluster = grid && ctx->solver_flow == VXP_SOLVER_CLUSTER && ctx->cluster_size > 0;
    const uint32_t flow = ctx->solver_flow == VXP_SOLVER_EVENTS ? 1u : 0u;
    WorldDev w = ctx->w.make(ctx->cfg, dt, phases, ctx->solver_div, device_pairs, margin, flow);
    const size_t smem = grid ? grid_smem(w.cache_cap) : block_smem(w.cache_cap);
    if (!grid) w.cfg.block_smem = (uint32_t)smem;
    w.cfg.flow_smem_chunks = grid ? flow_chunks(solve_smem()) : 0u;
    w.cfg.heavy_voxels = ctx->heavy_voxels;
    w.cfg.count_bricks = ctx->count_bricks ? 1u : 0u;
    w.cfg.owner_groups = cluster ? ctx->cluster_size : 1u;
    if (ctx->record_substeps) {
        const size_t need = (size_t)std::max(1u, ctx->cfg.substeps) * std::max(1u, ctx->w.n_bodies) * 13u;
        if (ctx->subrec.reserve(need) != cudaSuccess) return fail(ctx, VXP_ERR_OOM, "substep record buffer");
        w.cfg.record_substeps = 1u;
        w.subrec = ctx->subrec.p;
    }
    CK(cudaMemcpyAsync(ctx->d_world.p, &w, sizeof(w), cudaMemcpyHostToDevice, ctx->stream));
    const ColliderSet cs = ctx->cols.set();
    CK(cudaEventRecord(ctx->ev0, ctx->stream));
    if (grid) {
        CK(cudaMemsetAsync(ctx->bar.p, 0, 3 * sizeof(GridBar), ctx->stream));
        const WorldDev* wp = ctx->d_world.p;
        GridBar* bp = ctx->bar.p;
        const unsigned long long timeout = ctx->wait_limit_ns ? ctx->wait_limit_ns : kGridWaitNs;
        void* args[] = {(void*)&wp, (void*)&cs, (void*)&bp, (void*)&timeout};
        CK(cudaLaunchCooperativeKernel((const void*)k_step_grid, dim3(ctx->grid_blocks), dim3(kGridThreads), args,
                                       smem, ctx->stream));
        CK(cudaEventRecord(ctx->ev_mid, ctx->stream));
        const uint32_t whole = cluster && ctx->cluster_whole ? 1u : 0u;
        if (!whole) {
            uint32_t part = cluster ? SOLVE_CONSTRAINTS : SOLVE_ALL;
            void* sargs[] = {(void*)&wp, (void*)&bp, (void*)&timeout, (void*)&part};
            CK(cudaLaunchCooperativeKernel((const void*)k_solve_grid, dim3(ctx->grid_blocks), dim3(kSolveThreads),
                                           sargs, solve_smem(), ctx->stream));
        }
        if (cluster) {
            CK(cudaEventRecord(ctx->ev_cons, ctx->stream));
            cudaLaunchConfig_t lc = {};
            cudaLaunchAttribute at[1];
            cluster_config(&lc, at, ctx->cluster_size, ctx->cluster_smem, ctx->stream);
            CK(cudaLaunchKernelEx(&lc, k_solve_cluster, wp, std::min(ctx->cluster_smem, ctx->cluster_state_cap),
                                  whole));
        }
    } else {
        k_step_block<kBlockThreads><<<1, kBlockThreads, smem, ctx->stream>>>(ctx->d_world.p, cs);
        CK(cudaGetLastError());
    }
    CK(cudaEventRecord(ctx->ev1, ctx->stream));
    ctx->last_grid = grid;
    ctx->last_cluster = cluster;
    if (device_pairs && !ctx->count_pending) {
        CK(cudaMemcpyAsync(ctx->h_count, ctx->w.n_pairs_dev.p, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                           ctx->stream));
        CK(cudaEventRecord(ctx->ev_count, ctx->stream));
        ctx->count_pending = true;
    }
    return VXP_OK;
}

int check_device_error(vxp_ctx* ctx) {
    CK(cudaStreamSynchronize(ctx->stream));
    return ctx->w.take_error(ctx->stream, ctx->err);
}

// The pair list of the current body state into ctx->w.pairs (host waits).
int compute_device_pairs(vxp_ctx* ctx, float margin, uint32_t* n_out) {
    if (int rc = ctx->cols.sync(ctx->stream, ctx->err)) return rc;
    WorldBuffers& w = ctx->w;
    const uint32_t n = w.n_bodies;
    const ColliderSet cs = ctx->cols.set();
    if (n == 0) {
        *n_out = 0;
        return VXP_OK;
    }
    if (ctx->pair_counts.reserve(w.body_cap) != cudaSuccess || ctx->pair_offsets.reserve(w.body_cap) != cudaSuccess)
        return fail(ctx, VXP_ERR_OOM, "pair scratch");
    const uint32_t tb = 256, nb = (n + tb - 1) / tb;
    const uint32_t wb = (n * 32u + tb - 1) / tb;
    k_body_aabbs<<<nb, tb, 0, ctx->stream>>>(w.body.p, w.prop.p, n, cs, margin, w.aabb_mn.p, w.aabb_mx.p);
    uint32_t* masks = n <= w.bp_rows ? w.bpmask.p : nullptr;
    k_pairs<<<wb, tb, 0, ctx->stream>>>(w.ids.p, w.prop.p, n, w.aabb_mn.p, w.aabb_mx.p, ctx->pair_counts.p, nullptr,
                                        nullptr, 0, 0, masks, w.bp_stride);
    k_scan1<<<1, 1024, 0, ctx->stream>>>(ctx->pair_counts.p, ctx->pair_offsets.p, n, w.n_pairs_dev.p);
    CK(cudaGetLastError());
    // the write pass runs at once into the pair buffers as they are (it
    // writes no pair past their capacity); only when the total does not fit
    // are they grown and the pass run again
    auto write_pass = [&]() {
        k_pairs<<<wb, tb, 0, ctx->stream>>>(w.ids.p, w.prop.p, n, w.aabb_mn.p, w.aabb_mx.p, nullptr,
                                            ctx->pair_offsets.p, w.pairs.p, w.pair_cap, 1, masks, w.bp_stride);
        return cudaGetLastError();
    };
    const bool early = w.pairs.p != nullptr && w.pair_cap > 0u;
    if (early) CK(write_pass());
    uint32_t total = 0;
    CK(cudaMemcpyAsync(&total, w.n_pairs_dev.p, sizeof(total), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (!early || total > w.pair_cap) {
        if (int rc = w.ensure_pairs(total, ctx->err)) return rc;
        CK(write_pass());
    }
    *n_out = total;
    return VXP_OK;
}

}  // namespace

// ===========================================================================
// Allocation-free pair source (vxp_pairs_noalloc)
// ===========================================================================
// Some callers cannot let a library allocate device memory: an engine that
// runs its physics step on a frame thread where cudaMalloc's implicit device
// synchronisation would blow the frame budget, or one whose device memory is
// all handed out by its own allocator.  vxp_pairs_noalloc lets them run the
// broad-phase pair source on their own buffers: its only scratch (world
// AABBs, per-row pair counts and offsets, the total) is this file-scope
// array, sized for kNoAllocMaxBodies bodies, which every GPU that loads the
// library holds until the process exits.
constexpr uint32_t kNoAllocMaxBodies = 16384;
constexpr size_t kNoAllocScratchBytes = (size_t)kNoAllocMaxBodies * (2 * sizeof(float4) + 2 * sizeof(uint32_t)) + 256;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

struct NoAllocScratch {
    float4* mn;
    float4* mx;
    uint32_t* counts;
    uint32_t* offsets;
    uint32_t* total;
    uint32_t* unordered;  // set by the scan when ids are not strictly ascending
};
__host__ __device__ inline NoAllocScratch noalloc_layout(unsigned char* base) {
    NoAllocScratch s;
    s.mn = reinterpret_cast<float4*>(base);
    s.mx = s.mn + kNoAllocMaxBodies;
    s.counts = reinterpret_cast<uint32_t*>(s.mx + kNoAllocMaxBodies);
    s.offsets = s.counts + kNoAllocMaxBodies;
    s.total = s.offsets + kNoAllocMaxBodies;
    s.unordered = s.total + 1;
    return s;
}

// World AABB of each body's local AABB (AABB.transform, math.zig:686-693)
// inflated by margin; an empty local AABB (min > max) stands for a body
// without collider, whose box is its position.
__global__ void k_noalloc_aabbs(const float4* pos, const float4* rot, const float4* laabb, uint32_t n, float margin,
                                unsigned char* base) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const NoAllocScratch s = noalloc_layout(base);
    const F3 x = f3of(pos[i]);
    const Qt q = qof(rot[i]);
    const float4 lo4 = laabb[2 * i], hi4 = laabb[2 * i + 1];
    F3 lo, hi;
    if (lo4.x <= hi4.x && lo4.y <= hi4.y && lo4.z <= hi4.z) {
        const float inf = __int_as_float(0x7f800000);
        lo = F3{inf, inf, inf};
        hi = F3{-inf, -inf, -inf};
        for (int k = 0; k < 8; ++k) {
            const F3 corner{(k & 1) ? hi4.x : lo4.x, (k & 2) ? hi4.y : lo4.y, (k & 4) ? hi4.z : lo4.z};
            const F3 p = transform_point(x, q, corner);
            lo = min3(lo, p);
            hi = max3(hi, p);
        }
    } else {
        lo = x;
        hi = x;
    }
    lo = lo - F3{margin, margin, margin};
    hi = hi + F3{margin, margin, margin};
    s.mn[i] = make_float4(lo.x, lo.y, lo.z, 0.f);
    s.mx[i] = make_float4(hi.x, hi.y, hi.z, 0.f);
}

// Same sweep as k_pairs over caller arrays (ids ascending, so row order is id
// order).  Pass 0 counts per row, pass 1 writes at the scanned offsets.
__global__ void k_noalloc_pairs(const uint32_t* ids, const uint32_t* types, uint32_t n, unsigned char* base,
                                uint2* out, uint32_t cap, int pass) {
    const uint32_t sidx = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31;
    if (sidx >= n) return;
    const NoAllocScratch s = noalloc_layout(base);
    if (pass && *s.unordered) return;  // rejected by the scan: nothing is written
    const float4 a0 = s.mn[sidx], a1 = s.mx[sidx];
    const bool si = types[sidx] == 0u;
    const uint32_t id_s = ids[sidx];
    uint32_t o = pass ? s.offsets[sidx] : 0u;
    uint32_t cnt = 0;
    for (uint32_t t0 = sidx + 1; t0 < n; t0 += 32u) {
        const uint32_t t = t0 + lane;
        bool hit = false;
        if (t < n && !(si && types[t] == 0u)) {
            const float4 b0 = s.mn[t], b1 = s.mx[t];
            hit = a0.x <= b1.x && a1.x >= b0.x && a0.y <= b1.y && a1.y >= b0.y && a0.z <= b1.z && a1.z >= b0.z;
        }
        const uint32_t m = __ballot_sync(0xffffffffu, hit);
        if (pass && hit) {
            const uint32_t slot = o + __popc(m & ((1u << lane) - 1u));
            if (slot < cap) out[slot] = make_uint2(id_s, ids[t]);
        }
        o += __popc(m);
        cnt += __popc(m);
    }
    if (!pass && lane == 0) s.counts[sidx] = cnt;
}

// Exclusive scan of the per-row counts; also checks the ids' precondition
// (strictly ascending): when it fails, the total is 0, the flag word is set
// and the write pass writes nothing.
__global__ void __launch_bounds__(1024) k_noalloc_scan(uint32_t n, const uint32_t* ids, unsigned char* base,
                                                        uint32_t* count_out) {
    const NoAllocScratch s = noalloc_layout(base);
    uint32_t carry = 0;
    int bad = 0;
    for (uint32_t t0 = 0; t0 < n; t0 += blockDim.x) {
        const uint32_t i = t0 + threadIdx.x;
        const uint32_t v = i < n ? s.counts[i] : 0u;
        if (i + 1 < n && ids[i] >= ids[i + 1]) bad = 1;
        uint32_t tile;
        const uint32_t ex = block_excl_scan(v, &tile);
        if (i < n) s.offsets[i] = carry + ex;
        carry += tile;
    }
    bad = __syncthreads_or(bad);
    if (threadIdx.x == 0) {
        *s.unordered = bad ? 1u : 0u;
        *s.total = bad ? 0u : carry;
        *count_out = bad ? 0u : carry;
    }
}

namespace {
// Device address of g_noalloc_scratch, looked up once per device with that
// device current (a host-side mention of the array names a host stand-in,
// not device memory).  The address is kept for the life of the process, so
// the device must not be reset (cudaDeviceReset) while the library is loaded:
// the next call would hand the kernels the old context's address.
std::mutex g_noalloc_mu;
unsigned char* g_noalloc_addr[256] = {};

bool check_args_enabled() {
    static const bool on = [] {
        const char* v = std::getenv("VXP_CHECK_ARGS");
        return v && v[0] == '1';
    }();
    return on;
}

int noalloc_scratch_for_current_device(unsigned char** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) return VXP_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return VXP_ERR_CUDA;
        g_noalloc_addr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_noalloc_addr[dev];
    return VXP_OK;
}
}  // namespace

// ===========================================================================
// C ABI: single world
// ===========================================================================
extern "C" {

int vxp_abi_version(void) { return VXP_ABI_VERSION; }

void vxp_config_default(vxp_config* c) {
    std::memset(c, 0, sizeof(*c));
    c->gravity[0] = 0.0f;
    c->gravity[1] = -9.81f;
    c->gravity[2] = 0.0f;
    c->fixed_timestep = 1.0f / 60.0f;
    c->enable_sleeping = 1;
    c->enable_warm_starting = 1;
    c->substeps = 4;
    c->velocity_iterations = 1;
    c->position_iterations = 2;
    c->disable_rotation = 0;
    c->hertz = 30.0f;
    c->damping_ratio = 1.0f;
    c->position_correction_rate = 0.2f;
    c->max_position_correction = 0.04f;
    c->slop = 0.005f;
    c->warm_starting = 1;
    c->warm_start_scale = 0.8f;
    c->enable_friction = 1;
    c->enable_restitution = 1;
    c->use_brick_sat = 1;
    c->use_brick_pair_cache = 1;
    c->brick_pair_cache_size = 1024;
    c->reference_caps = 0;
    c->colouring = VXP_COLOUR_PROJECT;
    c->enable_islands = 1;
    c->max_bodies = 0;
    c->max_pairs = 0;
}

static int set_kernel_smem(uint32_t cache_cap) {
    if (cudaFuncSetAttribute(k_step_block<256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)block_smem(kMaxCacheSmem)) != cudaSuccess ||
        cudaFuncSetAttribute(k_step_block<512>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)block_smem(kMaxCacheSmem)) != cudaSuccess ||
        cudaFuncSetAttribute(k_step_grid, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)grid_smem(cache_cap)) != cudaSuccess ||
        cudaFuncSetAttribute(k_solve_grid, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)solve_smem()) !=
            cudaSuccess)
        return VXP_ERR_CUDA;
    return VXP_OK;
}

int vxp_create(const vxp_config* cfg, int device, vxp_ctx** out) {
    if (!cfg || !out) return VXP_ERR_ARG;
    *out = nullptr;
    if (cfg->substeps == 0) return VXP_ERR_ARG;
    if (cfg->position_iterations > 16) return VXP_ERR_ARG;
    if (cfg->brick_pair_cache_size > kMaxCacheSmem) return VXP_ERR_ARG;
    vxp_ctx* ctx = new vxp_ctx;
    ctx->cfg = *cfg;
    ctx->device = device;
    auto bail = [&](int rc) {
        vxp_destroy(ctx);
        return rc;
    };
    if (cudaSetDevice(device) != cudaSuccess) return bail(VXP_ERR_CUDA);
    int smc = 0;
    if (cudaDeviceGetAttribute(&smc, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return bail(VXP_ERR_CUDA);
    ctx->sm_count = smc;
    // A blocking stream: buffers are zero-filled (cudaMemset) and uploaded
    // (cudaMemcpy from pageable memory) on the legacy default stream, and
    // both can return before the device is done; a blocking stream orders
    // every kernel after that work.
    if (cudaStreamCreate(&ctx->stream) != cudaSuccess) return bail(VXP_ERR_CUDA);
    if (cudaEventCreate(&ctx->ev_start) != cudaSuccess || cudaEventCreate(&ctx->ev0) != cudaSuccess ||
        cudaEventCreate(&ctx->ev1) != cudaSuccess || cudaEventCreate(&ctx->ev_mid) != cudaSuccess ||
        cudaEventCreate(&ctx->ev_cons) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->ev_count, cudaEventDisableTiming) != cudaSuccess)
        return bail(VXP_ERR_CUDA);
    if (cudaMallocHost(&ctx->h_count, sizeof(uint32_t)) != cudaSuccess) return bail(VXP_ERR_OOM);
    *ctx->h_count = 0;
    const uint32_t cache_cap = cfg->brick_pair_cache_size ? cfg->brick_pair_cache_size : 1024u;
    if (set_kernel_smem(cache_cap)) return bail(VXP_ERR_CUDA);
    int per_sm = 0;
    int per_sm_solve = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_step_grid, kGridThreads, grid_smem(cache_cap)) !=
            cudaSuccess ||
        per_sm < 1 ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_solve, k_solve_grid, kSolveThreads, solve_smem()) !=
            cudaSuccess ||
        per_sm_solve < 1)
        return bail(VXP_ERR_CUDA);
    ctx->grid_blocks = (uint32_t)smc;  // one CTA per SM for both grid kernels
    // the largest cluster the device schedules for the sweeps: 16 CTAs (a
    // non-portable size), else 8; none leaves the grid solver in charge
    // each of its CTAs takes all the shared memory one block may have (the
    // state of the sweeps lives there)
    int optin = 0;
    cudaFuncAttributes fa = {};
    if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) == cudaSuccess &&
        cudaFuncGetAttributes(&fa, k_solve_cluster) == cudaSuccess && optin > (int)fa.sharedSizeBytes)
        ctx->cluster_smem = (uint32_t)(optin - (int)fa.sharedSizeBytes);
    cudaFuncSetAttribute(k_solve_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    cudaFuncSetAttribute(k_solve_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ctx->cluster_smem);
    for (uint32_t n : {16u, 8u}) {
        cudaLaunchConfig_t lc = {};
        cudaLaunchAttribute at[1];
        cluster_config(&lc, at, n, ctx->cluster_smem, ctx->stream);
        int active = 0;
        if (cudaOccupancyMaxActiveClusters(&active, k_solve_cluster, &lc) == cudaSuccess && active >= 1) {
            ctx->cluster_size = n;
            break;
        }
    }
    cudaGetLastError();  // a refused size is not an error of this context
    ctx->solver_flow = ctx->cluster_size ? VXP_SOLVER_CLUSTER : VXP_SOLVER_EVENTS;
    ctx->w.spill_rows = true;
    if (ctx->w.init(cache_cap, ctx->grid_blocks, ctx->err)) return bail(VXP_ERR_OOM);
    if (ctx->d_world.reserve(1) != cudaSuccess || ctx->bar.reserve(3) != cudaSuccess) return bail(VXP_ERR_OOM);
    if (ctx->w.ensure_pairs(std::max<uint32_t>(cfg->max_pairs, 1024), ctx->err)) return bail(VXP_ERR_OOM);
    if (ctx->w.ensure_bodies(std::max<uint32_t>(cfg->max_bodies, 256), ctx->err)) return bail(VXP_ERR_OOM);
    if (cudaDeviceSynchronize() != cudaSuccess) return bail(VXP_ERR_CUDA);
    *out = ctx;
    return VXP_OK;
}

void vxp_destroy(vxp_ctx* ctx) {
    if (!ctx) return;
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->ev_start) cudaEventDestroy(ctx->ev_start);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->ev_mid) cudaEventDestroy(ctx->ev_mid);
    if (ctx->ev_cons) cudaEventDestroy(ctx->ev_cons);
    if (ctx->ev_count) cudaEventDestroy(ctx->ev_count);
    if (ctx->h_count) cudaFreeHost(ctx->h_count);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

int vxp_last_error(const vxp_ctx* ctx, char* buf, size_t n) {
    if (!ctx || !buf || n == 0) return VXP_ERR_ARG;
    std::snprintf(buf, n, "%s", ctx->err.c_str());
    return VXP_OK;
}

int vxp_collider_upload(vxp_ctx* ctx, uint32_t collider_id, float voxel_size, const vxp_brick* bricks,
                        uint32_t n_bricks) {
    if (!ctx) return VXP_ERR_ARG;
    return ctx->cols.upload(collider_id, voxel_size, bricks, n_bricks, ctx->err);
}

int vxp_collider_edit(vxp_ctx* ctx, uint32_t collider_id, const int32_t* coords, const uint8_t* values, uint32_t n,
                      int mode) {
    if (!ctx) return VXP_ERR_ARG;
    if (mode != VXP_EDIT_SET && mode != VXP_EDIT_OCCUPANCY) return fail(ctx, VXP_ERR_ARG, "unknown edit mode %d", mode);
    return ctx->cols.edit(collider_id, coords, values, n, (uint32_t)mode, ctx->stream, ctx->err);
}

int vxp_collider_read(vxp_ctx* ctx, uint32_t collider_id, vxp_collider_info* info, vxp_brick* bricks, uint32_t cap,
                      uint32_t* n_bricks) {
    if (!ctx) return VXP_ERR_ARG;
    if (int rc = check_device_error(ctx)) return rc;
    return ctx->cols.read(collider_id, info, bricks, cap, n_bricks, ctx->stream, ctx->err);
}

int vxp_invalidate_cache_for_body(vxp_ctx* ctx, uint32_t body_id, uint32_t* n_invalidated) {
    if (!ctx) return VXP_ERR_ARG;
    if (ctx->d_word.reserve(1) != cudaSuccess) return fail(ctx, VXP_ERR_OOM, "device allocation failed");
    const uint32_t cap = ctx->w.cache_cap;
    CK(cudaMemsetAsync(ctx->d_word.p, 0, sizeof(uint32_t), ctx->stream));
    k_cache_invalidate<<<(cap + 255) / 256, 256, 0, ctx->stream>>>(ctx->w.ckey.p, cap, body_id, ctx->d_word.p);
    CK(cudaGetLastError());
    if (n_invalidated) {
        CK(cudaMemcpyAsync(n_invalidated, ctx->d_word.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    return VXP_OK;
}

int vxp_bodies_set(vxp_ctx* ctx, const vxp_body* b, uint32_t n) {
    if (!ctx) return VXP_ERR_ARG;
    CK(cudaStreamSynchronize(ctx->stream));
    return ctx->w.set_bodies(b, n, ctx->cols, ctx->err);
}

// vxp_bodies_export / vxp_batch_world_export on one world's buffers.
static int export_world(WorldBuffers& w, const ColliderSet& cs, const vxp_state_view* dst, uint32_t first,
                        uint32_t n, int device_memory, void* consumer, cudaStream_t stream, int device,
                        std::string& err) {
    if (!dst) {
        err = "null state view";
        return VXP_ERR_ARG;
    }
    if (first > w.n_bodies || n > w.n_bodies - first) {
        err = fmt("bodies [%u, %u + %u) outside the %u bodies", first, first, n, w.n_bodies);
        return VXP_ERR_ARG;
    }
    // per field: the caller's pointer and its bytes
    void* ptr[7] = {dst->position, dst->rotation, dst->linear_velocity, dst->angular_velocity,
                    dst->aabb_min, dst->aabb_max, dst->sleeping};
    const size_t per[7] = {12, 16, 12, 12, 12, 12, 1};
    if (n == 0) return VXP_OK;
    const dim3 grid((n + 255u) / 256u);
    if (device_memory) {
        for (int f = 0; f < 7; ++f) {
            if (!ptr[f]) continue;
            cudaPointerAttributes at{};
            if (cudaPointerGetAttributes(&at, ptr[f]) != cudaSuccess ||
                (at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged) || at.device != device) {
                cudaGetLastError();  // an unregistered host pointer can leave this call's error behind
                err = fmt("state view field %d is not device memory of device %d", f, device);
                return VXP_ERR_ARG;
            }
        }
        k_export<<<grid, 256, 0, stream>>>(w.body.p, w.prop.p, first, n, cs, *dst);
        if (cudaPeekAtLastError() != cudaSuccess) {
            err = fmt("export launch: %s", cudaGetErrorString(cudaGetLastError()));
            return VXP_ERR_CUDA;
        }
        if (consumer) {
            cudaEvent_t ev = nullptr;
            if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess ||
                cudaEventRecord(ev, stream) != cudaSuccess ||
                cudaStreamWaitEvent((cudaStream_t)consumer, ev, 0) != cudaSuccess) {
                if (ev) cudaEventDestroy(ev);
                err = "export: consumer stream wait failed";
                return VXP_ERR_CUDA;
            }
            cudaEventDestroy(ev);  // released once the recorded work completes
        }
        return VXP_OK;
    }
    // host memory: every requested field into the staging buffer, then copied out
    size_t off[7], total = 0;
    for (int f = 0; f < 7; ++f) {
        off[f] = total;
        if (ptr[f]) total += (per[f] * n + 15u) & ~(size_t)15u;
    }
    if (total == 0) return VXP_OK;
    if (w.export_stage.reserve(total) != cudaSuccess) {
        err = "export staging: device allocation failed";
        return VXP_ERR_OOM;
    }
    unsigned char* st = w.export_stage.p;
    vxp_state_view dv{};
    dv.position = dst->position ? reinterpret_cast<float*>(st + off[0]) : nullptr;
    dv.rotation = dst->rotation ? reinterpret_cast<float*>(st + off[1]) : nullptr;
    dv.linear_velocity = dst->linear_velocity ? reinterpret_cast<float*>(st + off[2]) : nullptr;
    dv.angular_velocity = dst->angular_velocity ? reinterpret_cast<float*>(st + off[3]) : nullptr;
    dv.aabb_min = dst->aabb_min ? reinterpret_cast<float*>(st + off[4]) : nullptr;
    dv.aabb_max = dst->aabb_max ? reinterpret_cast<float*>(st + off[5]) : nullptr;
    dv.sleeping = dst->sleeping ? st + off[6] : nullptr;
    k_export<<<grid, 256, 0, stream>>>(w.body.p, w.prop.p, first, n, cs, dv);
    if (cudaPeekAtLastError() != cudaSuccess) {
        err = fmt("export launch: %s", cudaGetErrorString(cudaGetLastError()));
        return VXP_ERR_CUDA;
    }
    for (int f = 0; f < 7; ++f) {
        if (!ptr[f]) continue;
        if (cudaMemcpyAsync(ptr[f], st + off[f], per[f] * n, cudaMemcpyDeviceToHost, stream) != cudaSuccess) {
            err = "export: copy to host failed";
            return VXP_ERR_CUDA;
        }
    }
    if (cudaStreamSynchronize(stream) != cudaSuccess) {
        err = "export: stream synchronize failed";
        return VXP_ERR_CUDA;
    }
    return VXP_OK;
}

int vxp_bodies_export(vxp_ctx* ctx, const vxp_state_view* dst, uint32_t first, uint32_t n, int device_memory,
                      void* consumer_stream) {
    if (!ctx) return VXP_ERR_ARG;
    if (!device_memory) {
        if (int rc = check_device_error(ctx)) return rc;
    }
    if (int rc = ctx->cols.sync(ctx->stream, ctx->err)) return rc;
    return export_world(ctx->w, ctx->cols.set(), dst, first, n, device_memory, consumer_stream, ctx->stream,
                        ctx->device, ctx->err);
}

int vxp_bodies_get(vxp_ctx* ctx, vxp_body* b, uint32_t n) {
    if (!ctx || (!b && n)) return fail(ctx, VXP_ERR_ARG, "null argument");
    if (int rc = check_device_error(ctx)) return rc;
    return ctx->w.get_bodies(b, n, ctx->stream, ctx->err);
}

int vxp_mass_properties(float vs, const vxp_brick* bricks, uint32_t n, float density, float* inv_mass,
                        float inv_inertia[9]) {
    if ((!bricks && n) || !inv_mass || !inv_inertia) return VXP_ERR_ARG;
    std::vector<int32_t> pos((size_t)n * 3);
    std::vector<uint8_t> vox((size_t)n * 512);
    for (uint32_t i = 0; i < n; ++i) {
        for (int k = 0; k < 3; ++k) pos[(size_t)i * 3 + k] = bricks[i].pos[k];
        std::memcpy(&vox[(size_t)i * 512], bricks[i].voxels, 512);
    }
    ColliderMeta h;
    collider_metadata(vs, pos.data(), vox.data(), n, h);
    if (h.solid == 0) {
        *inv_mass = 0.0f;
        for (int k = 0; k < 9; ++k) inv_inertia[k] = 0.0f;
        return VXP_OK;
    }
    // body.zig:473-519 with getCenterOfMass (collider.zig:376-403)
    const float vv = vs * vs * vs;
    const float vm = vv * density;
    const float total = vm * (float)h.solid;
    float sum[3] = {0.f, 0.f, 0.f};
    uint32_t count = 0;
    const float half = vs * 0.5f;
    for (uint32_t b = 0; b < n; ++b)
        for (int i = 0; i < 512; ++i) {
            if ((vox[(size_t)b * 512 + i] & 7u) == 0u) continue;
            const int c[3] = {i % 8, (i / 8) % 8, i / 64};
            for (int k = 0; k < 3; ++k) {
                const float p = ((float)(pos[(size_t)b * 3 + k] * 8 + c[k]) * vs + half) + vs * 0.5f;
                sum[k] = sum[k] + p;
            }
            ++count;
        }
    const float inv_count = 1.0f / (float)count;
    const float com[3] = {sum[0] * inv_count, sum[1] * inv_count, sum[2] * inv_count};
    vxp::M33 I;
    for (int k = 0; k < 9; ++k) I.m[k] = 0.0f;
    for (uint32_t b = 0; b < n; ++b)
        for (int i = 0; i < 512; ++i) {
            if ((vox[(size_t)b * 512 + i] & 7u) == 0u) continue;
            const int c[3] = {i % 8, (i / 8) % 8, i / 64};
            float r[3];
            for (int k = 0; k < 3; ++k) {
                const float p = ((float)(pos[(size_t)b * 3 + k] * 8 + c[k]) * vs + half) + vs * 0.5f;
                r[k] = p - com[k];
            }
            const float r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
            I.m[0] += vm * (r2 - r[0] * r[0]);
            I.m[4] += vm * (r2 - r[1] * r[1]);
            I.m[8] += vm * (r2 - r[2] * r[2]);
            I.m[1] -= vm * r[0] * r[1];
            I.m[2] -= vm * r[0] * r[2];
            I.m[5] -= vm * r[1] * r[2];
        }
    I.m[3] = I.m[1];
    I.m[6] = I.m[2];
    I.m[7] = I.m[5];
    *inv_mass = 1.0f / total;
    const vxp::M33 inv = vxp::mat3_inverse(I);
    for (int k = 0; k < 9; ++k) inv_inertia[k] = inv.m[k];
    return VXP_OK;
}

int vxp_step(vxp_ctx* ctx, float dt, const vxp_pair* pairs, uint32_t n_pairs) {
    if (!ctx || (!pairs && n_pairs)) return fail(ctx, VXP_ERR_ARG, "null argument");
    if (int rc = ctx->w.ensure_pairs(n_pairs, ctx->err)) return rc;
    CK(cudaEventRecord(ctx->ev_start, ctx->stream));
    if (n_pairs)
        CK(cudaMemcpyAsync(ctx->w.pairs.p, pairs, n_pairs * sizeof(vxp_pair), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->w.n_pairs_dev.p, &n_pairs, sizeof(uint32_t), cudaMemcpyHostToDevice, ctx->stream));
    ctx->last_pairs = n_pairs;
    return launch_step(ctx, dt, PH_STEP, false, 0.0f);
}

int vxp_step_device_pairs(vxp_ctx* ctx, float dt, float margin) {
    if (!ctx) return VXP_ERR_ARG;
    // grow ahead of need from the pair count of an earlier step (copied back
    // without waiting); a list that still overflows leaves the step undone
    // and is reported as VXP_ERR_CAP at the next wait
    if (ctx->count_pending && cudaEventQuery(ctx->ev_count) == cudaSuccess) {
        ctx->count_pending = false;
        const uint32_t seen = *ctx->h_count;
        ctx->last_pairs = seen;
        if (seen > ctx->w.pair_cap - ctx->w.pair_cap / 4u) {
            CK(cudaStreamSynchronize(ctx->stream));
            if (int rc = ctx->w.ensure_pairs(seen + seen / 2u + 1024u, ctx->err)) return rc;
        }
    }
    CK(cudaEventRecord(ctx->ev_start, ctx->stream));
    return launch_step(ctx, dt, PH_STEP, true, margin);
}

// system.narrowPhase() alone: no all-sleeping early return (that test is
// VoxelPhysicsSystem.step's).
int vxp_narrow_phase(vxp_ctx* ctx, const vxp_pair* pairs, uint32_t n_pairs) {
    if (!ctx || (!pairs && n_pairs)) return fail(ctx, VXP_ERR_ARG, "null argument");
    if (int rc = ctx->w.ensure_pairs(n_pairs, ctx->err)) return rc;
    CK(cudaEventRecord(ctx->ev_start, ctx->stream));
    if (n_pairs)
        CK(cudaMemcpyAsync(ctx->w.pairs.p, pairs, n_pairs * sizeof(vxp_pair), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->w.n_pairs_dev.p, &n_pairs, sizeof(uint32_t), cudaMemcpyHostToDevice, ctx->stream));
    ctx->last_pairs = n_pairs;
    return launch_step(ctx, 0.0f, PH_NARROW, false, 0.0f);
}

// system.solve() + updateSleepStates on the manifolds of the last narrow phase.
int vxp_solve(vxp_ctx* ctx, float dt) {
    if (!ctx) return VXP_ERR_ARG;
    CK(cudaEventRecord(ctx->ev_start, ctx->stream));
    return launch_step(ctx, dt, PH_SOLVE, false, 0.0f);
}

int vxp_manifolds_get(vxp_ctx* ctx, vxp_manifold* out, uint32_t cap, uint32_t* n_out) {
    if (!ctx || !n_out) return VXP_ERR_ARG;
    if (int rc = check_device_error(ctx)) return rc;
    uint32_t fr[2];
    CK(cudaMemcpy(fr, ctx->w.frame.p, sizeof(fr), cudaMemcpyDeviceToHost));
    // the latest narrow phase wrote man[frame & 1] with fr[1] slots
    const uint32_t slot = fr[0] & 1u;
    const ManifoldRec* m = slot ? ctx->w.man1.p : ctx->w.man0.p;
    const uint32_t P = std::min<uint32_t>(fr[1], ctx->w.pair_cap);
    std::vector<ManifoldRec> hm(P);
    if (P) CK(cudaMemcpy(hm.data(), m, P * sizeof(ManifoldRec), cudaMemcpyDeviceToHost));
    uint32_t k = 0;
    for (uint32_t p = 0; p < P; ++p) {
        if (hm[p].n == 0u) continue;
        if (k < cap && out) {
            // slots past contact_count hold stale data on the device
            ManifoldRec r = hm[p];
            r._pad = 0u;
            for (uint32_t i = r.n; i < 4u; ++i) std::memset(&r.c[i], 0, sizeof(ContactRec));
            for (uint32_t i = 0; i < r.n; ++i) r.c[i]._pad = 0u;
            std::memcpy(&out[k], &r, sizeof(vxp_manifold));
        }
        ++k;
    }
    *n_out = k;
    return VXP_OK;
}

int vxp_set_candidate_dump(vxp_ctx* ctx, uint32_t capacity) {
    if (!ctx) return VXP_ERR_ARG;
    if (capacity && ctx->w.dump.reserve(capacity) != cudaSuccess) return fail(ctx, VXP_ERR_OOM, "dump buffer");
    ctx->w.dump_cap = capacity;
    return VXP_OK;
}

int vxp_candidates_get(vxp_ctx* ctx, vxp_candidate* out, uint32_t cap, uint32_t* n_out) {
    if (!ctx || !n_out) return VXP_ERR_ARG;
    if (int rc = check_device_error(ctx)) return rc;
    uint32_t n = 0;
    CK(cudaMemcpy(&n, ctx->w.ctr.p + C_DUMP_N, sizeof(n), cudaMemcpyDeviceToHost));
    *n_out = n;
    if (n > ctx->w.dump_cap) return fail(ctx, VXP_ERR_CAP, "candidate dump overflow: %u > %u", n, ctx->w.dump_cap);
    // cache-consulting pairs are detected speculatively while the cache is
    // replayed; the records of the pairs that hit are not part of the step
    static_assert(sizeof(WorldDev::Cand) == sizeof(vxp_candidate), "candidate layout");
    std::vector<vxp_candidate> all(n);
    if (n) CK(cudaMemcpy(all.data(), ctx->w.dump.p, n * sizeof(vxp_candidate), cudaMemcpyDeviceToHost));
    uint32_t P = 0;
    CK(cudaMemcpy(&P, ctx->w.frame.p + 1, sizeof(P), cudaMemcpyDeviceToHost));
    P = std::min<uint32_t>(P, ctx->w.pair_cap);
    std::vector<PairInfo> pi(P);
    if (P) CK(cudaMemcpy(pi.data(), ctx->w.pinfo.p, P * sizeof(PairInfo), cudaMemcpyDeviceToHost));
    uint32_t k = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t p = all[i].pair_index;
        if (p < P && (pi[p].flags & PF_CACHE) && pi[p].hit == 1u) continue;
        if (out && k < cap) out[k] = all[i];
        ++k;
    }
    *n_out = k;
    return VXP_OK;
}

int vxp_stats_get(vxp_ctx* ctx, vxp_stats* s) {
    if (!ctx || !s) return VXP_ERR_ARG;
    if (int rc = check_device_error(ctx)) return rc;
    return ctx->w.stats(s, ctx->last_pairs, ctx->stream, ctx->err);
}

int vxp_colours_get(vxp_ctx* ctx, uint32_t* colours, uint32_t cap, uint32_t* n_out) {
    if (!ctx || !n_out) return VXP_ERR_ARG;
    if (int rc = check_device_error(ctx)) return rc;
    uint32_t M = 0;
    CK(cudaMemcpy(&M, ctx->w.ctr.p + C_CONSTRAINTS, sizeof(M), cudaMemcpyDeviceToHost));
    *n_out = M;
    const uint32_t k = std::min(M, cap);
    if (k && colours) CK(cudaMemcpy(colours, ctx->w.colour.p, k * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    return VXP_OK;
}

int vxp_pairs_from_bodies(vxp_ctx* ctx, float margin, vxp_pair* out, uint32_t cap, uint32_t* n_out) {
    if (!ctx || !n_out) return VXP_ERR_ARG;
    uint32_t n = 0;
    if (int rc = compute_device_pairs(ctx, margin, &n)) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    *n_out = n;
    const uint32_t k = std::min(n, cap);
    if (k && out) CK(cudaMemcpy(out, ctx->w.pairs.p, k * sizeof(vxp_pair), cudaMemcpyDeviceToHost));
    return n > cap ? fail(ctx, VXP_ERR_CAP, "pair output holds %u, need %u", cap, n) : VXP_OK;
}

int vxp_last_step_ms(vxp_ctx* ctx, float out[3]) {
    if (!ctx || !out) return VXP_ERR_ARG;
    CK(cudaStreamSynchronize(ctx->stream));
    float a = 0.f, b = 0.f, c = 0.f;
    CK(cudaEventElapsedTime(&a, ctx->ev_start, ctx->ev0));
    CK(cudaEventElapsedTime(&b, ctx->ev0, ctx->ev1));
    CK(cudaEventElapsedTime(&c, ctx->ev_start, ctx->ev1));
    out[0] = a;
    out[1] = b;
    out[2] = c;
    return VXP_OK;
}

// See the allocation-free section above and include/vxp.h.
int vxp_pairs_noalloc(const float* positions, const float* rotations, const float* local_aabbs, const uint32_t* ids,
                      const uint32_t* body_types, uint32_t n, float margin, vxp_pair* out, uint32_t cap,
                      uint32_t* count, void* stream) {
    if (n > kNoAllocMaxBodies) return VXP_ERR_CAP;
    if (!count || (n && (!positions || !rotations || !local_aabbs || !ids || !body_types)) || (cap && !out))
        return VXP_ERR_ARG;
    // An error the caller left pending is theirs: launch nothing and leave it
    // in place rather than report it later as this call's failure.
    if (cudaPeekAtLastError() != cudaSuccess) return VXP_ERR_CUDA;
    unsigned char* base = nullptr;
    if (int rc = noalloc_scratch_for_current_device(&base)) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (n == 0) {
        return cudaMemsetAsync(count, 0, sizeof(uint32_t), st) == cudaSuccess ? VXP_OK : VXP_ERR_CUDA;
    }
    const uint32_t tb = 256, nb = (n + tb - 1) / tb, wb = (n * 32u + tb - 1) / tb;
    k_noalloc_aabbs<<<nb, tb, 0, st>>>(reinterpret_cast<const float4*>(positions),
                                       reinterpret_cast<const float4*>(rotations),
                                       reinterpret_cast<const float4*>(local_aabbs), n, margin, base);
    k_noalloc_pairs<<<wb, tb, 0, st>>>(ids, body_types, n, base, nullptr, 0, 0);
    k_noalloc_scan<<<1, 1024, 0, st>>>(n, ids, base, count);
    k_noalloc_pairs<<<wb, tb, 0, st>>>(ids, body_types, n, base, reinterpret_cast<uint2*>(out), cap, 1);
    if (cudaPeekAtLastError() != cudaSuccess) {
        (void)cudaGetLastError();  // this call's launch error: reported here, so cleared
        return VXP_ERR_CUDA;
    }
    // With VXP_CHECK_ARGS=1 in the environment the call also waits for its
    // work and turns ids that are not strictly ascending into VXP_ERR_ARG;
    // otherwise such a call only leaves *count at 0 and writes no pair.
    if (check_args_enabled()) {
        uint32_t unordered = 0;
        if (cudaStreamSynchronize(st) != cudaSuccess) return VXP_ERR_CUDA;
        if (cudaMemcpy(&unordered, noalloc_layout(base).unordered, sizeof(unordered), cudaMemcpyDeviceToHost) !=
            cudaSuccess)
            return VXP_ERR_CUDA;
        if (unordered) return VXP_ERR_ARG;
    }
    return VXP_OK;
}

// Phase boundaries of the last step, ns since its start (diagnostics).
int vxp_phase_times(vxp_ctx* ctx, uint64_t* out, uint32_t n) {
    if (!ctx || !out) return VXP_ERR_ARG;
    CK(cudaStreamSynchronize(ctx->stream));
    unsigned long long t[TS_N];
    CK(cudaMemcpy(t, ctx->w.ts.p, sizeof(t), cudaMemcpyDeviceToHost));
    for (uint32_t i = 0; i < n && i < TS_N; ++i) out[i] = t[i] >= t[0] ? (uint64_t)(t[i] - t[0]) : 0u;
    return VXP_OK;
}

int vxp_snapshot_substeps(vxp_ctx* ctx, int enable) {
    if (!ctx) return VXP_ERR_ARG;
    ctx->record_substeps = enable != 0;
    return VXP_OK;
}

int vxp_substeps_get(vxp_ctx* ctx, float* out, uint32_t cap_floats, uint32_t* n_substeps) {
    if (!ctx || !n_substeps || (!out && cap_floats)) return VXP_ERR_ARG;
    if (int rc = check_device_error(ctx)) return rc;
    uint32_t ns = 0;
    CK(cudaMemcpy(&ns, ctx->w.ctr.p + C_SUBREC, sizeof(ns), cudaMemcpyDeviceToHost));
    if (!ctx->record_substeps || !ctx->subrec.p) ns = 0;
    const size_t need = (size_t)ns * ctx->w.n_bodies * 13u;
    if (need > cap_floats) return fail(ctx, VXP_ERR_ARG, "substep record needs %zu floats", need);
    if (need) CK(cudaMemcpy(out, ctx->subrec.p, need * sizeof(float), cudaMemcpyDeviceToHost));
    *n_substeps = ns;
    return VXP_OK;
}

int vxp_last_kernel_ms(vxp_ctx* ctx, float out[2]) {
    if (!ctx || !out) return VXP_ERR_ARG;
    CK(cudaEventSynchronize(ctx->ev1));
    if (ctx->last_grid) {
        CK(cudaEventElapsedTime(&out[0], ctx->ev0, ctx->ev_mid));
        CK(cudaEventElapsedTime(&out[1], ctx->ev_mid, ctx->ev1));
    } else {
        CK(cudaEventElapsedTime(&out[0], ctx->ev0, ctx->ev1));
        out[1] = 0.0f;
    }
    return VXP_OK;
}

int vxp_last_solve_split_ms(vxp_ctx* ctx, float out[2]) {
    if (!ctx || !out) return VXP_ERR_ARG;
    CK(cudaEventSynchronize(ctx->ev1));
    if (ctx->last_cluster) {
        CK(cudaEventElapsedTime(&out[0], ctx->ev_mid, ctx->ev_cons));
        CK(cudaEventElapsedTime(&out[1], ctx->ev_cons, ctx->ev1));
    } else {
        out[0] = 0.0f;
        out[1] = 0.0f;
    }
    return VXP_OK;
}

int vxp_set_traffic_accounting(vxp_ctx* ctx, int on) {
    if (!ctx) return VXP_ERR_ARG;
    ctx->count_bricks = on != 0;
    return VXP_OK;
}

int vxp_set_cluster_constraints(vxp_ctx* ctx, int on) {
    if (!ctx) return VXP_ERR_ARG;
    ctx->cluster_whole = on != 0;
    return VXP_OK;
}

int vxp_set_cluster_shared_bytes(vxp_ctx* ctx, uint32_t bytes) {
    if (!ctx) return VXP_ERR_ARG;
    ctx->cluster_state_cap = bytes;
    return VXP_OK;
}

int vxp_cluster_size(vxp_ctx* ctx, uint32_t* n) {
    if (!ctx || !n) return VXP_ERR_ARG;
    *n = ctx->cluster_size;
    return VXP_OK;
}

int vxp_synchronize(vxp_ctx* ctx) {
    if (!ctx) return VXP_ERR_ARG;
    return check_device_error(ctx);
}

int vxp_set_launch_mode(vxp_ctx* ctx, int mode) {
    if (!ctx || mode < -1 || mode > 1) return VXP_ERR_ARG;
    ctx->use_grid = mode;
    return VXP_OK;
}

int vxp_set_solver_blocks_divisor(vxp_ctx* ctx, uint32_t div) {
    if (!ctx || div == 0) return VXP_ERR_ARG;
    ctx->solver_div = div;
    return VXP_OK;
}

int vxp_set_heavy_pair_voxels(vxp_ctx* ctx, uint32_t n) {
    if (!ctx) return VXP_ERR_ARG;
    ctx->heavy_voxels = n;
    return VXP_OK;
}

int vxp_set_wait_limit_ns(vxp_ctx* ctx, uint64_t ns) {
    if (!ctx) return VXP_ERR_ARG;
    ctx->wait_limit_ns = ns;
    return VXP_OK;
}

int vxp_set_probe_tables(vxp_ctx* ctx, int enable) {
    if (!ctx) return VXP_ERR_ARG;
    ctx->cols.set_tables(enable != 0);
    return VXP_OK;
}

int vxp_set_solver_mode(vxp_ctx* ctx, uint32_t mode) {
    if (!ctx || mode > VXP_SOLVER_CLUSTER) return VXP_ERR_ARG;
    if (mode == VXP_SOLVER_CLUSTER && ctx->cluster_size == 0) return VXP_ERR_STATE;
    ctx->solver_flow = mode;
    return VXP_OK;
}

}  // extern "C"

// ===========================================================================
// Batched worlds
// ===========================================================================
// Many independent worlds advance together: one launch of k_step_block, block
// b stepping the b-th world of the launch order with the whole step (pair
// source, narrow phase, solver) inside the CTA.  The launch is captured once
// in a CUDA graph and replayed every step.  Each world's arithmetic does not
// depend on the launch shape, so every schedule gives the same bits.
struct vxp_batch {
    vxp_config cfg;
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    ColliderStore cols;
    std::vector<std::unique_ptr<WorldBuffers>> slots;
    std::vector<uint8_t> active;
    std::vector<float> est_ms;        // last measured step time per slot
    std::vector<uint32_t> order;      // launch position -> slot
    DBuf<WorldDev> d_worlds;
    DBuf<unsigned long long> d_ts;    // per launch position: [start, end]
    DBuf<uint32_t> d_status;          // per launch position: [error word, pair count]
    uint32_t threads = 256;           // CTA size
    uint32_t order_mode = 1;          // 0: slot order, 1: longest measured / largest first
    // per-world tiles: > 0, worlds of at least this many bodies step as
    // 512-thread CTAs (launch positions [0, n_big)) and the rest as 256-thread
    // CTAs, two launches side by side in the graph (second stream)
    uint32_t tile_min_bodies = 0;
    uint32_t n_big = 0;
    cudaStream_t stream2 = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    uint32_t graph_tile = 0, graph_nbig = 0;
    float margin = 0.1f;
    float built_dt = -1.0f;
    bool rebuild = true;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    const void* graph_worlds = nullptr;  // what the graph's launch was captured with
    ColliderSet graph_cs{};
    uint32_t graph_n = 0, graph_threads = 0;
    DBuf<uint32_t> d_word;  // a count read back by the host
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    uint32_t cache_cap = 1024;
};

namespace {

int bfail(vxp_batch* b, int code, const char* f, ...) {
    if (b) {
        char buf[512];
        va_list ap;
        va_start(ap, f);
        vsnprintf(buf, sizeof(buf), f, ap);
        va_end(ap);
        b->err = buf;
    }
    return code;
}
#define BK(call)                                                                                          \
    do {                                                                                                  \
        cudaError_t e_ = (call);                                                                          \
        if (e_ != cudaSuccess) return bfail(bt, VXP_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

__global__ void k_batch_times(const WorldDev* worlds, uint32_t n, unsigned long long* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const unsigned long long* ts = worlds[i].ts;
    out[2 * i] = ts[TS_START];
    out[2 * i + 1] = ts[TS_END] > ts[TS_START] ? ts[TS_END] : ts[TS_START];
}

// Per launch position: the world's sticky error word and its pair count of
// the last step, gathered so the host reads every world with one copy.
__global__ void k_batch_status(const WorldDev* worlds, uint32_t n, uint32_t* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[2 * i] = worlds[i].ctr[C_ERROR];
    out[2 * i + 1] = *worlds[i].n_pairs_dev;
}

// Launch order, device WorldDev array and the graph of one step.
int batch_prepare(vxp_batch* bt, float dt) {
    if (int rc = bt->cols.sync(bt->stream, bt->err)) return rc;
    if (bt->rebuild || dt != bt->built_dt) {
        std::vector<uint32_t> ord;
        for (uint32_t s = 0; s < bt->slots.size(); ++s)
            if (bt->active[s] && bt->slots[s]) ord.push_back(s);
        if (bt->order_mode == 1) {
            std::stable_sort(ord.begin(), ord.end(), [&](uint32_t a, uint32_t c) {
                const float ea = bt->est_ms[a] > 0 ? bt->est_ms[a] : 1e-6f * (float)bt->slots[a]->n_bodies;
                const float ec = bt->est_ms[c] > 0 ? bt->est_ms[c] : 1e-6f * (float)bt->slots[c]->n_bodies;
                return ea > ec;
            });
        }
        if (bt->tile_min_bodies) {
            // the 512-thread worlds first, each group in the order above
            const auto mid = std::stable_partition(ord.begin(), ord.end(), [&](uint32_t x) {
                return bt->slots[x]->n_bodies >= bt->tile_min_bodies;
            });
            bt->n_big = (uint32_t)(mid - ord.begin());
        } else {
            bt->n_big = bt->threads == 512 ? (uint32_t)ord.size() : 0u;
        }
        bt->order = ord;
        std::vector<WorldDev> wd(ord.size());
        for (size_t i = 0; i < ord.size(); ++i)
        {
            wd[i] = bt->slots[ord[i]]->make(bt->cfg, dt, PH_STEP, 128, true, bt->margin, 0u);
            wd[i].cfg.block_smem = (uint32_t)block_smem(bt->cache_cap);
        }
        if (bt->d_worlds.reserve(std::max<size_t>(wd.size(), 1)) != cudaSuccess ||
            bt->d_ts.reserve(2 * std::max<size_t>(wd.size(), 1)) != cudaSuccess ||
            bt->d_status.reserve(2 * std::max<size_t>(wd.size(), 1)) != cudaSuccess)
            return bfail(bt, VXP_ERR_OOM, "batch world table");
        if (!wd.empty())
            BK(cudaMemcpyAsync(bt->d_worlds.p, wd.data(), wd.size() * sizeof(WorldDev), cudaMemcpyHostToDevice,
                               bt->stream));
        BK(cudaStreamSynchronize(bt->stream));
        bt->built_dt = dt;
        bt->rebuild = false;
    }
    const ColliderSet cs = bt->cols.set();
    const uint32_t n = (uint32_t)bt->order.size();
    if (bt->exec && bt->d_worlds.p == bt->graph_worlds && cs.c == bt->graph_cs.c &&
        cs.grid == bt->graph_cs.grid && cs.vox == bt->graph_cs.vox && cs.n == bt->graph_cs.n && cs.nb == bt->graph_cs.nb &&
        n == bt->graph_n && bt->threads == bt->graph_threads && bt->tile_min_bodies == bt->graph_tile &&
        bt->n_big == bt->graph_nbig)
        return VXP_OK;
    if (bt->exec) {
        cudaGraphExecDestroy(bt->exec);
        bt->exec = nullptr;
    }
    if (bt->graph) {
        cudaGraphDestroy(bt->graph);
        bt->graph = nullptr;
    }
    if (n == 0) return VXP_OK;
    const size_t smem = block_smem(bt->cache_cap);
    BK(cudaStreamBeginCapture(bt->stream, cudaStreamCaptureModeThreadLocal));
    if (bt->tile_min_bodies) {
        // 512-thread worlds on the batch stream, 256-thread worlds on the
        // second stream, forked from and joined back into the first
        const uint32_t nb = bt->n_big, ns = n - bt->n_big;
        const bool both = nb > 0 && ns > 0;
        if (both) {
            cudaEventRecord(bt->ev_fork, bt->stream);
            cudaStreamWaitEvent(bt->stream2, bt->ev_fork, 0);
        }
        if (nb)
            k_step_block<512><<<nb, 512, smem, bt->stream>>>(bt->d_worlds.p, cs);
        if (ns)
            k_step_block<256><<<ns, 256, smem, both ? bt->stream2 : bt->stream>>>(
                bt->d_worlds.p + nb, cs);
        if (both) {
            cudaEventRecord(bt->ev_join, bt->stream2);
            cudaStreamWaitEvent(bt->stream, bt->ev_join, 0);
        }
    } else if (bt->threads == 512) {
        k_step_block<512><<<n, 512, smem, bt->stream>>>(bt->d_worlds.p, cs);
    } else {
        k_step_block<256><<<n, 256, smem, bt->stream>>>(bt->d_worlds.p, cs);
    }
    const cudaError_t le = cudaGetLastError();
    cudaGraph_t g = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(bt->stream, &g);
    if (le != cudaSuccess || ce != cudaSuccess)
        return bfail(bt, VXP_ERR_CUDA, "graph capture: %s / %s", cudaGetErrorString(le), cudaGetErrorString(ce));
    bt->graph = g;
    BK(cudaGraphInstantiate(&bt->exec, bt->graph, 0));
    bt->graph_worlds = bt->d_worlds.p;
    bt->graph_cs = cs;
    bt->graph_n = n;
    bt->graph_threads = bt->threads;
    bt->graph_tile = bt->tile_min_bodies;
    bt->graph_nbig = bt->n_big;
    return VXP_OK;
}

}  // namespace

extern "C" {

int vxp_batch_create(const vxp_config* cfg, int device, uint32_t max_worlds, vxp_batch** out) {
    if (!cfg || !out || max_worlds == 0) return VXP_ERR_ARG;
    *out = nullptr;
    if (cfg->substeps == 0 || cfg->position_iterations > 16 || cfg->brick_pair_cache_size > kMaxCacheSmem)
        return VXP_ERR_ARG;
    vxp_batch* bt = new vxp_batch;
    bt->cfg = *cfg;
    bt->device = device;
    bt->cache_cap = cfg->brick_pair_cache_size ? cfg->brick_pair_cache_size : 1024u;
    bt->slots.resize(max_worlds);
    bt->active.assign(max_worlds, 0);
    bt->est_ms.assign(max_worlds, 0.0f);
    auto bail = [&](int rc) {
        vxp_batch_destroy(bt);
        return rc;
    };
    if (cudaSetDevice(device) != cudaSuccess) return bail(VXP_ERR_CUDA);
    // blocking, for the same reason as a context's stream (vxp_create)
    if (cudaStreamCreate(&bt->stream) != cudaSuccess || cudaStreamCreate(&bt->stream2) != cudaSuccess)
        return bail(VXP_ERR_CUDA);
    if (cudaEventCreate(&bt->ev0) != cudaSuccess || cudaEventCreate(&bt->ev1) != cudaSuccess ||
        cudaEventCreateWithFlags(&bt->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&bt->ev_join, cudaEventDisableTiming) != cudaSuccess)
        return bail(VXP_ERR_CUDA);
    if (set_kernel_smem(bt->cache_cap)) return bail(VXP_ERR_CUDA);
    *out = bt;
    return VXP_OK;
}

void vxp_batch_destroy(vxp_batch* bt) {
    if (!bt) return;
    if (bt->stream) cudaStreamSynchronize(bt->stream);
    if (bt->exec) cudaGraphExecDestroy(bt->exec);
    if (bt->graph) cudaGraphDestroy(bt->graph);
    if (bt->ev0) cudaEventDestroy(bt->ev0);
    if (bt->ev1) cudaEventDestroy(bt->ev1);
    if (bt->ev_fork) cudaEventDestroy(bt->ev_fork);
    if (bt->ev_join) cudaEventDestroy(bt->ev_join);
    if (bt->stream2) cudaStreamDestroy(bt->stream2);
    if (bt->stream) cudaStreamDestroy(bt->stream);
    delete bt;
}

int vxp_batch_last_error(const vxp_batch* bt, char* buf, size_t n) {
    if (!bt || !buf || n == 0) return VXP_ERR_ARG;
    std::snprintf(buf, n, "%s", bt->err.c_str());
    return VXP_OK;
}

int vxp_batch_collider_upload(vxp_batch* bt, uint32_t collider_id, float voxel_size, const vxp_brick* bricks,
                              uint32_t n_bricks) {
    if (!bt) return VXP_ERR_ARG;
    BK(cudaStreamSynchronize(bt->stream));
    return bt->cols.upload(collider_id, voxel_size, bricks, n_bricks, bt->err);
}

int vxp_batch_collider_edit(vxp_batch* bt, uint32_t collider_id, const int32_t* coords, const uint8_t* values,
                            uint32_t n, int mode) {
    if (!bt) return VXP_ERR_ARG;
    if (mode != VXP_EDIT_SET && mode != VXP_EDIT_OCCUPANCY) return bfail(bt, VXP_ERR_ARG, "unknown edit mode %d", mode);
    return bt->cols.edit(collider_id, coords, values, n, (uint32_t)mode, bt->stream, bt->err);
}

int vxp_batch_collider_read(vxp_batch* bt, uint32_t collider_id, vxp_collider_info* info, vxp_brick* bricks,
                            uint32_t cap, uint32_t* n_bricks) {
    if (!bt) return VXP_ERR_ARG;
    return bt->cols.read(collider_id, info, bricks, cap, n_bricks, bt->stream, bt->err);
}

int vxp_batch_invalidate_cache_for_body(vxp_batch* bt, uint32_t world, uint32_t body_id, uint32_t* n_invalidated) {
    if (!bt || world >= bt->slots.size() || !bt->slots[world]) return bfail(bt, VXP_ERR_ARG, "no such world");
    if (bt->d_word.reserve(1) != cudaSuccess) return bfail(bt, VXP_ERR_OOM, "device allocation failed");
    WorldBuffers& w = *bt->slots[world];
    const uint32_t cap = w.cache_cap;
    BK(cudaMemsetAsync(bt->d_word.p, 0, sizeof(uint32_t), bt->stream));
    k_cache_invalidate<<<(cap + 255) / 256, 256, 0, bt->stream>>>(w.ckey.p, cap, body_id, bt->d_word.p);
    BK(cudaGetLastError());
    if (n_invalidated) {
        BK(cudaMemcpyAsync(n_invalidated, bt->d_word.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, bt->stream));
        BK(cudaStreamSynchronize(bt->stream));
    }
    return VXP_OK;
}

int vxp_batch_world_set(vxp_batch* bt, uint32_t world, const vxp_body* bodies, uint32_t n, uint32_t pair_capacity) {
    if (!bt || world >= bt->slots.size()) return bfail(bt, VXP_ERR_ARG, "world index out of range");
    BK(cudaStreamSynchronize(bt->stream));
    auto& slot = bt->slots[world];
    // a fresh world starts with an empty contact manager and cache; a slot
    // that held an earlier world keeps its buffers (no allocation, no free,
    // which would wait for the whole device) and starts from them zeroed
    if (slot) {
        BK(slot->zero_all(bt->stream));
        BK(cudaStreamSynchronize(bt->stream));
        slot->n_bodies = 0;
        slot->collider_public.clear();
    } else {
        slot.reset(new WorldBuffers);
    }
    slot->live = true;
    if (int rc = slot->init(bt->cache_cap, 1, bt->err)) return rc;
    if (int rc = slot->set_bodies(bodies, n, bt->cols, bt->err)) return rc;
    const uint32_t want = pair_capacity ? pair_capacity : std::max<uint32_t>(1024, 16u * n);
    if (int rc = slot->ensure_pairs(want, bt->err)) return rc;
    bt->active[world] = n ? 1 : 0;
    bt->est_ms[world] = 0.0f;
    bt->rebuild = true;
    return VXP_OK;
}

int vxp_batch_world_clear(vxp_batch* bt, uint32_t world) {
    if (!bt || world >= bt->slots.size()) return bfail(bt, VXP_ERR_ARG, "world index out of range");
    BK(cudaStreamSynchronize(bt->stream));
    if (bt->slots[world]) bt->slots[world]->live = false;
    bt->active[world] = 0;
    bt->rebuild = true;
    return VXP_OK;
}

int vxp_batch_world_release(vxp_batch* bt, uint32_t world) {
    if (!bt || world >= bt->slots.size()) return bfail(bt, VXP_ERR_ARG, "world index out of range");
    BK(cudaStreamSynchronize(bt->stream));
    bt->slots[world].reset();
    bt->active[world] = 0;
    bt->rebuild = true;
    return VXP_OK;
}

int vxp_batch_world_get(vxp_batch* bt, uint32_t world, vxp_body* bodies, uint32_t n) {
    if (!bt || world >= bt->slots.size() || !bt->slots[world] || !bt->slots[world]->live)
        return bfail(bt, VXP_ERR_ARG, "no such world");
    BK(cudaStreamSynchronize(bt->stream));
    return bt->slots[world]->get_bodies(bodies, n, bt->stream, bt->err);
}

int vxp_batch_world_export(vxp_batch* bt, uint32_t world, const vxp_state_view* dst, uint32_t first, uint32_t n,
                           int device_memory, void* consumer_stream) {
    if (!bt || world >= bt->slots.size() || !bt->slots[world] || !bt->slots[world]->live)
        return bfail(bt, VXP_ERR_ARG, "no such world");
    if (!device_memory) BK(cudaStreamSynchronize(bt->stream));
    if (int rc = bt->cols.sync(bt->stream, bt->err)) return rc;
    return export_world(*bt->slots[world], bt->cols.set(), dst, first, n, device_memory, consumer_stream, bt->stream,
                        bt->device, bt->err);
}

int vxp_batch_world_stats(vxp_batch* bt, uint32_t world, vxp_stats* s) {
    if (!bt || !s || world >= bt->slots.size() || !bt->slots[world] || !bt->slots[world]->live)
        return bfail(bt, VXP_ERR_ARG, "no such world");
    BK(cudaStreamSynchronize(bt->stream));
    uint32_t np = 0;
    BK(cudaMemcpy(&np, bt->slots[world]->n_pairs_dev.p, sizeof(np), cudaMemcpyDeviceToHost));
    return bt->slots[world]->stats(s, np, bt->stream, bt->err);
}

uint64_t vxp_batch_world_bytes(vxp_batch* bt, uint32_t world) {
    if (!bt || world >= bt->slots.size() || !bt->slots[world]) return 0;
    return bt->slots[world]->device_bytes();
}

int vxp_batch_step(vxp_batch* bt, float dt, uint32_t n_steps) {
    if (!bt) return VXP_ERR_ARG;
    if (int rc = batch_prepare(bt, dt)) return rc;
    if (!bt->exec) return VXP_OK;
    BK(cudaEventRecord(bt->ev0, bt->stream));
    for (uint32_t s = 0; s < n_steps; ++s) BK(cudaGraphLaunch(bt->exec, bt->stream));
    BK(cudaEventRecord(bt->ev1, bt->stream));
    return VXP_OK;
}

// Waits; per-world errors; grows worlds whose pair list came close to (or
// over) capacity.  VXP_ERR_CAP: some world left its last step undone.
int vxp_batch_synchronize(vxp_batch* bt) {
    if (!bt) return VXP_ERR_ARG;
    BK(cudaStreamSynchronize(bt->stream));
    // every stepped world's error word and pair count in one read
    const uint32_t k = (uint32_t)bt->order.size();
    std::vector<uint32_t> st(2 * (size_t)k);
    if (k && bt->d_status.p && !bt->rebuild) {
        k_batch_status<<<(k + 127) / 128, 128, 0, bt->stream>>>(bt->d_worlds.p, k, bt->d_status.p);
        BK(cudaGetLastError());
        BK(cudaMemcpyAsync(st.data(), bt->d_status.p, st.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                           bt->stream));
        BK(cudaStreamSynchronize(bt->stream));
    }
    int rc = VXP_OK;
    if (bt->rebuild) {
        // worlds changed since the last step: the launch table may name
        // buffers that are gone, so read each current world directly
        for (uint32_t s = 0; s < bt->slots.size(); ++s) {
            if (!bt->active[s] || !bt->slots[s]) continue;
            WorldBuffers& w = *bt->slots[s];
            std::string e;
            const int r = w.take_error(bt->stream, e);
            if (r != VXP_OK && rc == VXP_OK) {
                rc = r;
                bt->err = fmt("world %u: %s", s, e.c_str());
            }
        }
        return rc;
    }
    for (uint32_t i = 0; i < k; ++i) {
        const uint32_t s = bt->order[i];
        if (!bt->active[s] || !bt->slots[s]) continue;
        WorldBuffers& w = *bt->slots[s];
        const uint32_t np = st[2 * i + 1];
        if (np > w.pair_cap - w.pair_cap / 4u) {
            if (int g = w.ensure_pairs(np + np / 2u + 1024u, bt->err)) return g;
            bt->rebuild = true;
        }
        if (st[2 * i] != 0u) {
            std::string e;
            const int r = w.take_error(bt->stream, e);
            if (r != VXP_OK && rc == VXP_OK) {
                rc = r;
                bt->err = fmt("world %u: %s", s, e.c_str());
            }
        }
    }
    return rc;
}

// Device time of the last step call (ms) and, per world, of its own CTA in
// the last step (ms, indexed by world slot; 0 for empty slots).
int vxp_batch_times(vxp_batch* bt, float* total_ms, float* world_ms, uint32_t n) {
    if (!bt) return VXP_ERR_ARG;
    BK(cudaStreamSynchronize(bt->stream));
    if (total_ms) BK(cudaEventElapsedTime(total_ms, bt->ev0, bt->ev1));
    const uint32_t k = (uint32_t)bt->order.size();
    if (k) {
        k_batch_times<<<(k + 127) / 128, 128, 0, bt->stream>>>(bt->d_worlds.p, k, bt->d_ts.p);
        std::vector<unsigned long long> t(2 * k);
        BK(cudaMemcpyAsync(t.data(), bt->d_ts.p, t.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                           bt->stream));
        BK(cudaStreamSynchronize(bt->stream));
        for (uint32_t i = 0; i < k; ++i) {
            const float ms = (float)(t[2 * i + 1] - t[2 * i]) * 1e-6f;
            bt->est_ms[bt->order[i]] = ms;
        }
    }
    if (world_ms)
        for (uint32_t s = 0; s < n && s < bt->slots.size(); ++s) world_ms[s] = bt->active[s] ? bt->est_ms[s] : 0.0f;
    return VXP_OK;
}

// Launch schedule: CTA size (256 or 512) and world order (0 slot order,
// 1 longest-first by the last measured world time, else by body count).
int vxp_batch_set_schedule(vxp_batch* bt, uint32_t threads, uint32_t order_mode) {
    if (!bt || (threads != 256 && threads != 512) || order_mode > 1) return VXP_ERR_ARG;
    bt->threads = threads;
    bt->order_mode = order_mode;
    bt->tile_min_bodies = 0;
    bt->rebuild = true;
    return VXP_OK;
}

int vxp_batch_set_tiles(vxp_batch* bt, uint32_t min_bodies_512, uint32_t order_mode) {
    if (!bt || min_bodies_512 == 0 || order_mode > 1) return VXP_ERR_ARG;
    bt->tile_min_bodies = min_bodies_512;
    bt->order_mode = order_mode;
    bt->rebuild = true;
    return VXP_OK;
}

// Schedule i of the autotuner: 0-3 one CTA size for every world, (256, slot
// order), (256, longest first), (512, slot order), (512, longest first);
// 4-7 per-world tiles, worlds of at least 128 / 256 / 512 / 1024 bodies as
// 512-thread CTAs and the rest as 256-thread CTAs, longest first.
static int batch_schedule(vxp_batch* bt, uint32_t i) {
    if (i < 4) return vxp_batch_set_schedule(bt, i < 2 ? 256u : 512u, i & 1u);
    return vxp_batch_set_tiles(bt, 128u << (i - 4u), 1u);
}

// Tries each schedule for trial_steps real steps (each world's results do
// not depend on the schedule) and keeps the fastest.  ms_out receives the
// mean step time of each of the VXP_BATCH_SCHEDULES schedules; *choice the
// index kept.
int vxp_batch_autotune(vxp_batch* bt, float dt, uint32_t trial_steps, float* ms_out, uint32_t* choice) {
    if (!bt || trial_steps == 0) return VXP_ERR_ARG;
    float best = 1e30f;
    uint32_t best_i = 0;
    for (uint32_t i = 0; i < VXP_BATCH_SCHEDULES; ++i) {
        if (int rc = batch_schedule(bt, i)) return rc;
        if (int rc = vxp_batch_step(bt, dt, 1)) return rc;  // measures world times, builds the graph
        if (int rc = vxp_batch_synchronize(bt)) return rc;
        if (int rc = vxp_batch_times(bt, nullptr, nullptr, 0)) return rc;
        bt->rebuild = true;  // re-sort with the measured times
        if (int rc = vxp_batch_step(bt, dt, trial_steps)) return rc;
        if (int rc = vxp_batch_synchronize(bt)) return rc;
        float ms = 0.f;
        if (int rc = vxp_batch_times(bt, &ms, nullptr, 0)) return rc;
        ms /= (float)trial_steps;
        if (ms_out) ms_out[i] = ms;
        if (ms < best) {
            best = ms;
            best_i = i;
        }
    }
    if (choice) *choice = best_i;
    return batch_schedule(bt, best_i);
}

}  // extern "C"
