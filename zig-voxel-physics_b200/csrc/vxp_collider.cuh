// Collider edits on the device: destructible and growing voxel bodies.
//
// An edit batch writes voxels of one uploaded collider, in one of two modes:
//   * set: each listed voxel gets the CollisionVoxel byte given, as
//     VoxelCollider.setCollisionVoxel stores it (src/collider.zig:267-273);
//   * occupancy: each listed voxel becomes solid or empty, then every listed
//     voxel and each of its six face neighbours that is solid is re-typed by
//     classifyFromNeighbors (src/collision_voxel.zig:103-130, 194-235; the
//     reference's helper for typing a voxel from its face neighbours,
//     exported by src/physics.zig:52) of the new occupancy.
// Then the collider's metadata is recomputed (VoxelCollider.recomputeMetadata,
// src/collider.zig:90-133, 283-333) and its neighbourhood-mask table rebuilt
// where it changed.  That is the sequence of reference calls an engine with
// destructible voxels makes on the host between steps; here it runs where the
// voxels already are, on the context's stream, without a host round trip.
// The host lists each coordinate once, with the last value the batch writes
// to its voxel byte (a brick reached through a shared hashBrickPos gives one
// byte several coordinates), and places new bricks before the edit runs, so
// every listed voxel has a brick.
#pragma once

#include "vxp_step.cuh"

namespace vxp {

enum : uint32_t { EDIT_SET = 0u, EDIT_OCCUPANCY = 1u };

// One CTA's share of the metadata, and the last CTA's ticket.
struct MetaPartial {
    int32_t mn[3], mx[3];
    float fmn[3], fmx[3];
    uint32_t solid, _pad;
};
constexpr uint32_t kMetaBlocks = 148;
constexpr uint32_t kMetaThreads = 256;
struct EditScratch {
    MetaPartial part[kMetaBlocks];
    uint32_t ticket;  // CTAs done (the last one resets it)
    uint32_t full;    // the table needs a full rebuild (bounds or range changed)
};

// Mutable byte of voxel (x, y, z) of collider c, or nullptr when its brick
// cell is outside the grid or holds no brick (the grid resolves each cell by
// hashBrickPos, as getOrCreateBrick / getBrick do, collider.zig:232-248).
__device__ __forceinline__ uint8_t* voxel_ptr(const DCollider& c, const int32_t* grid, uint8_t* vox, int32_t x,
                                              int32_t y, int32_t z) {
    const int32_t bx = (x >> 3) - c.bmin[0], by = (y >> 3) - c.bmin[1], bz = (z >> 3) - c.bmin[2];
    if ((uint32_t)bx >= (uint32_t)c.bdim[0] || (uint32_t)by >= (uint32_t)c.bdim[1] ||
        (uint32_t)bz >= (uint32_t)c.bdim[2])
        return nullptr;
    const int32_t slot = grid[c.grid_off + (uint32_t)(bx + c.bdim[0] * (by + c.bdim[1] * bz))];
    if (slot < 0) return nullptr;
    return vox + (size_t)(c.brick_off + (uint32_t)slot) * 512u + (uint32_t)((x & 7) + 8 * (y & 7) + 64 * (z & 7));
}

// classifyVoxel (collision_voxel.zig:194-210) of a solid voxel with the given
// empty-face mask (bit 0 -x, 1 +x, 2 -y, 3 +y, 4 -z, 5 +z): the type by the
// count of empty faces, the normal by computeNormalIndex (collision_voxel.zig:
// 103-130): the NORMAL_LUT entry equal to the sum of the empty faces'
// directions, or, when the sum is zero (opposite faces empty),
// findClosestNormalIndex of the zero vector, whose dot products all tie at 0,
// so entry 0.  No empty face is entry 0 as well.
__device__ __forceinline__ uint8_t classify_solid(uint32_t mask) {
    const uint32_t cnt = (uint32_t)__popc(mask);
    const uint32_t type = cnt == 0u ? kInside : (cnt == 1u ? kFace : (cnt == 2u ? kEdge : kCorner));
    auto code = [](uint32_t neg, uint32_t pos) { return neg == pos ? 0u : (pos ? 1u : 2u); };
    const uint32_t want = code(mask & 1u, (mask >> 1) & 1u) | (code((mask >> 2) & 1u, (mask >> 3) & 1u) << 2) |
                          (code((mask >> 4) & 1u, (mask >> 5) & 1u) << 4);
    // NORMAL_LUT as 2-bit codes per axis (1: +1, 2: -1), the table lut_normal decodes
    const uint32_t kCode[26] = {0x01, 0x02, 0x04, 0x08, 0x10, 0x20, 0x05, 0x09, 0x06, 0x0A, 0x11, 0x21, 0x12,
                                0x22, 0x14, 0x24, 0x18, 0x28, 0x15, 0x25, 0x19, 0x29, 0x16, 0x26, 0x1A, 0x2A};
    uint32_t normal = 0u;
    for (uint32_t i = 0; i < 26u; ++i)
        if (kCode[i] == want) normal = i;
    return (uint8_t)(type | (normal << 3));
}

// Step 1: each listed voxel's new byte (set mode), or its occupancy
// (occupancy mode: an empty voxel made solid holds a provisional inside byte
// until step 2; a solid voxel keeps its byte until then).  One thread per edit.
__global__ void k_edit_apply(const DCollider* cols, uint32_t ci, const int32_t* grid, uint8_t* vox,
                             const int4* edits, uint32_t n, uint32_t mode) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const DCollider c = cols[ci];
    const int4 e = edits[i];
    uint8_t* p = voxel_ptr(c, grid, vox, e.x, e.y, e.z);
    if (!p) return;  // the host placed every listed voxel's brick
    if (mode == EDIT_SET) *p = (uint8_t)e.w;
    else if (e.w == 0) *p = 0u;
    else if ((*p & 7u) == 0u) *p = (uint8_t)kInside;
}

// Step 2 (occupancy mode): every listed voxel and each face neighbour that is
// solid becomes classifyFromNeighbors of the new occupancy; a neighbour
// outside every brick is empty, as getCollisionVoxel returns.  stride 7: one
// thread per (edit, voxel or face neighbour), for colliders whose every voxel
// byte has one coordinate, so that threads writing the same byte write the
// same value; stride 1: one thread per listed voxel, the host having kept one
// coordinate per byte.  No thread changes a voxel's occupancy, which is all
// that any thread reads.
__global__ void k_edit_classify(const DCollider* cols, uint32_t ci, const int32_t* grid, uint8_t* vox,
                                const int4* edits, uint32_t n, uint32_t stride) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * stride) return;
    const DCollider c = cols[ci];
    const int4 e = edits[t / stride];
    const int32_t off[7][3] = {{0, 0, 0}, {-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
    const uint32_t k = t % stride;
    const int32_t x = e.x + off[k][0], y = e.y + off[k][1], z = e.z + off[k][2];
    uint8_t* p = voxel_ptr(c, grid, vox, x, y, z);
    if (!p || (*(volatile uint8_t*)p & 7u) == 0u) return;  // empty stays empty
    uint32_t mask = 0u;
    for (uint32_t f = 1; f < 7u; ++f) {
        const uint8_t* q = voxel_ptr(c, grid, vox, x + off[f][0], y + off[f][1], z + off[f][2]);
        if (!q || (*(volatile const uint8_t*)q & 7u) == 0u) mask |= 1u << (f - 1u);
    }
    *p = classify_solid(mask);
}

// Step 3: recomputeMetadata over the collider's bricks.  The bounds and the
// box are minima and maxima and the count a sum, so any order gives the
// reference's result: min_bound / max_bound over the solid voxels (max
// exclusive), the local AABB over the (brick_pos * 8 + coord) * vs boxes of
// the solid voxels, the solid count; zero bounds when nothing is solid.  Each
// thread reads 16 voxel bytes at a time; each CTA leaves a partial, and the
// last CTA to finish merges them, writes the collider and decides the table:
// its own range when the new probe centres fit nb_cap entries, else none; a
// full rebuild when the bounds or the range changed, or when `full` asks.
__global__ void __launch_bounds__(kMetaThreads) k_edit_meta(DCollider* cols, uint32_t ci, const uint8_t* vox,
                                                            const int4* bpos, EditScratch* sc, uint32_t full) {
    __shared__ int32_t s_mn[3], s_mx[3];
    __shared__ float s_fmn[3][kMetaThreads / 32], s_fmx[3][kMetaThreads / 32];
    __shared__ uint32_t s_solid, s_last;
    const uint32_t tid = threadIdx.x, lane = tid & 31u, wid = tid >> 5;
    const float vs = cols[ci].vs;
    const uint32_t brick_off = cols[ci].brick_off, n_bricks = cols[ci].n_bricks;
    if (tid < 3) {
        s_mn[tid] = INT32_MAX;
        s_mx[tid] = INT32_MIN;
    }
    if (tid == 0) s_solid = 0u;
    __syncthreads();
    const float inf = __int_as_float(0x7f800000);
    int32_t mn[3] = {INT32_MAX, INT32_MAX, INT32_MAX}, mx[3] = {INT32_MIN, INT32_MIN, INT32_MIN};
    float fmn[3] = {inf, inf, inf}, fmx[3] = {-inf, -inf, -inf};
    uint32_t solid = 0u;
    const uint4* v16 = reinterpret_cast<const uint4*>(vox + (size_t)brick_off * 512u);
    const uint32_t chunks = n_bricks * 32u;
    for (uint32_t q = blockIdx.x * blockDim.x + tid; q < chunks; q += gridDim.x * blockDim.x) {
        const uint4 w4 = v16[q];
        const uint32_t words[4] = {w4.x, w4.y, w4.z, w4.w};
        if ((words[0] | words[1] | words[2] | words[3]) == 0u) continue;
        const int4 bp = bpos[brick_off + (q >> 5)];
        const int32_t bb[3] = {bp.x, bp.y, bp.z};
        for (uint32_t j = 0; j < 16u; ++j) {
            if (((words[j >> 2] >> (8u * (j & 3u))) & 7u) == 0u) continue;
            ++solid;
            const uint32_t i = (q & 31u) * 16u + j;
            const int32_t cc[3] = {(int32_t)(i & 7u), (int32_t)((i >> 3) & 7u), (int32_t)(i >> 6)};
            for (int k = 0; k < 3; ++k) {
                const int32_t vc = bb[k] * 8 + cc[k];
                mn[k] = min(mn[k], vc);
                mx[k] = max(mx[k], vc + 1);
                const float lp = ((float)bb[k] * 8.0f + (float)cc[k]) * vs;
                fmn[k] = fminf(fmn[k], lp);
                fmx[k] = fmaxf(fmx[k], lp + vs);
            }
        }
    }
    solid = warp_sum(solid);
    for (int k = 0; k < 3; ++k)
        for (uint32_t d = 16; d > 0; d >>= 1) {
            mn[k] = min(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], d));
            mx[k] = max(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], d));
            fmn[k] = fminf(fmn[k], __shfl_xor_sync(0xffffffffu, fmn[k], d));
            fmx[k] = fmaxf(fmx[k], __shfl_xor_sync(0xffffffffu, fmx[k], d));
        }
    if (lane == 0) {
        atomicAdd(&s_solid, solid);
        for (int k = 0; k < 3; ++k) {
            atomicMin(&s_mn[k], mn[k]);
            atomicMax(&s_mx[k], mx[k]);
            s_fmn[k][wid] = fmn[k];
            s_fmx[k][wid] = fmx[k];
        }
    }
    __syncthreads();
    if (tid == 0) {
        MetaPartial& pp = sc->part[blockIdx.x];
        pp.solid = s_solid;
        for (int k = 0; k < 3; ++k) {
            float a = inf, b = -inf;
            for (uint32_t w = 0; w < blockDim.x / 32u; ++w) {
                a = fminf(a, s_fmn[k][w]);
                b = fmaxf(b, s_fmx[k][w]);
            }
            pp.mn[k] = s_mn[k];
            pp.mx[k] = s_mx[k];
            pp.fmn[k] = a;
            pp.fmx[k] = b;
        }
        __threadfence();
        s_last = atomicAdd(&sc->ticket, 1u) == gridDim.x - 1u;
    }
    __syncthreads();
    if (!s_last || tid != 0) return;
    __threadfence();
    uint32_t tot = 0u;
    int32_t gmn[3] = {INT32_MAX, INT32_MAX, INT32_MAX}, gmx[3] = {INT32_MIN, INT32_MIN, INT32_MIN};
    float gfmn[3] = {inf, inf, inf}, gfmx[3] = {-inf, -inf, -inf};
    for (uint32_t b = 0; b < gridDim.x; ++b) {
        const volatile MetaPartial& pp = sc->part[b];
        tot += pp.solid;
        for (int k = 0; k < 3; ++k) {
            gmn[k] = min(gmn[k], pp.mn[k]);
            gmx[k] = max(gmx[k], pp.mx[k]);
            gfmn[k] = fminf(gfmn[k], pp.fmn[k]);
            gfmx[k] = fmaxf(gfmx[k], pp.fmx[k]);
        }
    }
    DCollider& o = cols[ci];
    bool changed = false;
    uint64_t centres = 1u;
    for (int k = 0; k < 3; ++k) {
        const int32_t lo = tot ? gmn[k] : 0, hi = tot ? gmx[k] : 0;
        changed |= lo != o.min_bound[k] || hi != o.max_bound[k];
        o.min_bound[k] = lo;
        o.max_bound[k] = hi;
        o.aabb_min[k] = gfmn[k];
        o.aabb_max[k] = gfmx[k];
        centres *= (uint64_t)((int64_t)hi - lo + 2);
    }
    o.solid_count = tot;
    const uint32_t off = (o.nb_cap != 0u && centres <= o.nb_cap) ? o.nb_base : kNoTable;
    changed |= off != o.nb_off;
    o.nb_off = off;
    sc->full = (changed || full) ? 1u : 0u;
    sc->ticket = 0u;
}

// Step 4, when the bounds and the table range stayed: the table entries of
// the probe centres within 2 voxels of an edit (a centre reads the types of
// its 27 neighbours, and a type changes only within 1 voxel of an edit).
// One thread per (edit, centre offset in 5 x 5 x 5).
__global__ void k_edit_table_local(ColliderSet cs, uint4* nb, uint32_t ci, const int4* edits, uint32_t n,
                                   const EditScratch* sc) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * 125u || sc->full) return;
    const DCollider& c = cs.c[ci];
    if (c.nb_off == kNoTable) return;
    const int4 e = edits[t / 125u];
    const uint32_t o = t % 125u;
    const int32_t x = e.x + (int32_t)(o % 5u) - 2 - (c.min_bound[0] - 1),
                  y = e.y + (int32_t)((o / 5u) % 5u) - 2 - (c.min_bound[1] - 1),
                  z = e.z + (int32_t)(o / 25u) - 2 - (c.min_bound[2] - 1);
    const uint32_t ex = (uint32_t)(c.max_bound[0] - c.min_bound[0]) + 2u,
                   ey = (uint32_t)(c.max_bound[1] - c.min_bound[1]) + 2u,
                   ez = (uint32_t)(c.max_bound[2] - c.min_bound[2]) + 2u;
    if ((uint32_t)x >= ex || (uint32_t)y >= ey || (uint32_t)z >= ez) return;
    const uint32_t idx = (uint32_t)x + ex * ((uint32_t)y + ey * (uint32_t)z);
    nb[c.nb_off + idx] = nbhd_entry(cs, c, idx, ex, ey);
}

// Step 4, when the bounds or the table range changed: the whole table.
__global__ void k_edit_table_full(ColliderSet cs, uint4* nb, uint32_t ci, const EditScratch* sc) {
    if (!sc->full) return;
    const DCollider& c = cs.c[ci];
    if (c.nb_off == kNoTable) return;
    const uint32_t ex = (uint32_t)(c.max_bound[0] - c.min_bound[0]) + 2u,
                   ey = (uint32_t)(c.max_bound[1] - c.min_bound[1]) + 2u,
                   ez = (uint32_t)(c.max_bound[2] - c.min_bound[2]) + 2u;
    const uint32_t total = ex * ey * ez;
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x)
        nb[c.nb_off + e] = nbhd_entry(cs, c, e, ex, ey);
}

// BrickPairCache.invalidateBody (narrow_phase.zig:305-312): every valid entry
// whose key holds the body id becomes invalid; *count gains the number.
__global__ void k_cache_invalidate(CacheKeyRec* keys, uint32_t cap, uint32_t body_id, uint32_t* count) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t hit = 0u;
    if (i < cap) {
        CacheKeyRec& k = keys[i];
        if (k.valid && (k.a == body_id || k.b == body_id)) {
            k.valid = 0u;
            hit = 1u;
        }
    }
    hit = warp_sum(hit);
    if ((threadIdx.x & 31u) == 0u && hit) atomicAdd(count, hit);
}

}  // namespace vxp
