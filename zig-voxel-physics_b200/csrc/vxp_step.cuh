// vxp_step.cuh — the phases of one physics step on the device.
//
// Included by vxp_lib.cu only.  See vxp_world.cuh for the layouts and the
// phase map.  Float expressions keep the reference's operation order (the
// library is compiled with --fmad=false and IEEE div/sqrt).
#pragma once

#include <cstdint>

#include "vxp_math.cuh"
#include "vxp_world.cuh"

namespace vxp {

__device__ __forceinline__ F3 f3of(float4 a) { return F3{a.x, a.y, a.z}; }
__device__ __forceinline__ Qt qof(float4 a) { return Qt{a.x, a.y, a.z, a.w}; }
__device__ __forceinline__ float4 f4of(F3 a, float w) { return make_float4(a.x, a.y, a.z, w); }
__device__ __forceinline__ float4 f4of(Qt a) { return make_float4(a.x, a.y, a.z, a.w); }

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Ordered-int key of a float: min/max of keys == min/max of the floats.
__device__ __forceinline__ int32_t fkey(float f) {
    const int32_t i = __float_as_int(f);
    return i >= 0 ? i : (i ^ 0x7FFFFFFF);
}
__device__ __forceinline__ float fkey_inv(int32_t k) {
    return __int_as_float(k >= 0 ? k : (k ^ 0x7FFFFFFF));
}

// ---------------------------------------------------------------------------
// Groups
// ---------------------------------------------------------------------------
struct BlockGroup {
    // One CTA's barriers are cheap: the solver sweeps colour batch by colour
    // batch (the event-ordered sweeps are not compiled for this group).
    static constexpr bool kEventSweeps = false;
    static constexpr bool kDistributed = false;  // shared memory is the CTA's own
    __device__ uint32_t rank() const { return threadIdx.x; }
    __device__ uint32_t size() const { return blockDim.x; }
    __device__ uint32_t block() const { return 0; }
    __device__ uint32_t nblocks() const { return 1; }
    __device__ bool sync() {
        __syncthreads();
        return true;
    }
    // The solver runs on the same CTA.
    __device__ BlockGroup subgroup(uint32_t) const { return *this; }
    __device__ bool member() const { return true; }
};

struct GridBar {
    unsigned int count;
    unsigned int gen;
};

struct GridGroup {
    static constexpr bool kEventSweeps = true;
    static constexpr bool kDistributed = false;
    GridBar* bar;
    uint32_t* err;
    unsigned long long timeout_ns;
    uint32_t nb;        // participating blocks: base .. base + nb - 1
    uint32_t base = 0;
    __device__ uint32_t rank() const { return (blockIdx.x - base) * blockDim.x + threadIdx.x; }
    __device__ uint32_t size() const { return nb * blockDim.x; }
    __device__ uint32_t block() const { return blockIdx.x - base; }
    __device__ uint32_t nblocks() const { return nb; }
    __device__ bool member() const { return blockIdx.x - base < nb; }
    // The first k blocks, with their own barrier word (bar + 1): the solver's
    // colour batches are small, and a barrier over a few blocks costs far less
    // than one over the whole grid.  The other blocks leave the kernel, or
    // run as tail(k).
    __device__ GridGroup subgroup(uint32_t k) const { return GridGroup{bar + 1, err, timeout_ns, k, base}; }
    // The blocks after the first k, with the third barrier word (bar + 2).
    __device__ GridGroup tail(uint32_t k) const { return GridGroup{bar + 2, err, timeout_ns, nb - k, base + k}; }
    // Bounded grid barrier: a waiting block gives up after timeout_ns, sets
    // ERR_TIMEOUT and every later sync() of every block returns false.  The
    // block's threads meet at __syncthreads, then thread 0 arrives with an
    // acquire-release add on the count (the last to arrive resets it and
    // bumps the generation with a release add) and waits with acquire loads
    // of the generation: release / acquire at GPU scope, no full fence (a
    // sequentially consistent fence here was seen to stall one block for
    // hundreds of microseconds behind the memory traffic of a busy phase).
    __device__ bool sync() {
        __shared__ int s_ok;
        __syncthreads();
        if (threadIdx.x == 0) {
            int ok = 1;
            unsigned int g;
            asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(g) : "l"(&bar->gen) : "memory");
            unsigned int arrived;
            asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;" : "=r"(arrived) : "l"(&bar->count) : "memory");
            if (arrived == nb - 1) {
                asm volatile("st.relaxed.gpu.global.u32 [%0], 0;" ::"l"(&bar->count) : "memory");
                asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(&bar->gen) : "memory");
            } else {
                const unsigned long long t0 = global_ns();
                for (;;) {
                    unsigned int v;
                    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(&bar->gen) : "memory");
                    if (v != g) break;
                    __nanosleep(64);
                    if (global_ns() - t0 > timeout_ns) {
                        atomicOr(err, ERR_TIMEOUT);
                        ok = 0;
                        break;
                    }
                }
            }
            unsigned int e;
            asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(e) : "l"(err) : "memory");
            if (e & ERR_TIMEOUT) ok = 0;
            s_ok = ok;
        }
        __syncthreads();
        return s_ok != 0;
    }
};

// The CTAs of one thread-block cluster (the grid is exactly one cluster).
// sync() is the hardware cluster barrier (release / acquire at cluster scope,
// about 0.2 us for 16 CTAs against about 0.8 us for one flag handed between
// two SMs through L2).  That barrier cannot time out, so only code whose
// every block passes the same sequence of sync() calls runs on this group:
// the solver's colour sweeps and the store, whose barrier count depends only
// on values every block reads before the first barrier (see
// world_step_sweeps).  sync() never fails.
struct ClusterGroup {
    static constexpr bool kEventSweeps = false;
    static constexpr bool kDistributed = true;  // other CTAs' shared memory through mapa
    __device__ uint32_t rank() const { return blockIdx.x * blockDim.x + threadIdx.x; }
    __device__ uint32_t size() const { return gridDim.x * blockDim.x; }
    __device__ uint32_t block() const { return blockIdx.x; }
    __device__ uint32_t nblocks() const { return gridDim.x; }
    __device__ bool member() const { return true; }
    __device__ ClusterGroup subgroup(uint32_t) const { return *this; }
    __device__ bool sync() {
        asm volatile("barrier.cluster.arrive.release;\n\tbarrier.cluster.wait.acquire;" ::: "memory");
        return true;
    }
};

// ---------------------------------------------------------------------------
// Block-level primitives (blockDim.x <= 1024, multiple of 32)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v) {
    const uint32_t lane = threadIdx.x & 31;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t o = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= (uint32_t)d) v += o;
    }
    return v;
}
__device__ __forceinline__ uint32_t warp_sum(uint32_t v) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
    return v;
}
// Exclusive block scan; *total receives the block sum (all threads).
__device__ uint32_t block_excl_scan(uint32_t v, uint32_t* total) {
    __shared__ uint32_t s_w[33];
    const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const uint32_t inc = warp_incl_scan(v);
    if (lane == 31) s_w[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        const uint32_t x = lane < nw ? s_w[lane] : 0u;
        const uint32_t xi = warp_incl_scan(x);
        if (lane < nw) s_w[lane] = xi - x;
        if (lane == 31) s_w[32] = xi;
    }
    __syncthreads();
    const uint32_t r = s_w[wid] + inc - v;
    *total = s_w[32];
    __syncthreads();
    return r;
}
__device__ uint32_t block_sum(uint32_t v) {
    uint32_t t;
    block_excl_scan(v, &t);
    return t;
}

// Exclusive scan over the group of f(i), i in [0, n).  write(i, prefix) is
// called for every i; returns the total.  Uses scratch[nblocks].
template <class G, class F, class W>
__device__ bool group_scan(G& g, uint32_t n, F f, W write, uint32_t* scratch, uint32_t* total_out) {
    const uint32_t nb = g.nblocks(), b = g.block();
    const uint32_t seg = (n + nb - 1) / nb;
    const uint32_t lo = min(n, b * seg), hi = min(n, lo + seg);
    uint32_t part = 0;
    for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) part += f(i);
    part = block_sum(part);
    if (threadIdx.x == 0) scratch[b] = part;
    if (!g.sync()) return false;
    uint32_t base = 0, tot = 0;
    for (uint32_t j = threadIdx.x; j < nb; j += blockDim.x) {
        const uint32_t x = *(volatile uint32_t*)&scratch[j];
        tot += x;
        if (j < b) base += x;
    }
    base = block_sum(base);
    tot = block_sum(tot);
    uint32_t carry = base;
    for (uint32_t t0 = lo; t0 < hi; t0 += blockDim.x) {
        const uint32_t i = t0 + threadIdx.x;
        const uint32_t v = i < hi ? f(i) : 0u;
        uint32_t tile;
        const uint32_t ex = block_excl_scan(v, &tile);
        if (i < hi) write(i, carry + ex);
        carry += tile;
    }
    *total_out = tot;
    return g.sync();
}

// ---------------------------------------------------------------------------
// Collider access
// ---------------------------------------------------------------------------
struct ColliderSet {
    const DCollider* c;
    const int32_t* grid;
    const uint8_t* vox;
    uint32_t n;
    const uint4* nb;  // neighbourhood masks (DCollider::nb_off)
};

__device__ __forceinline__ uint32_t voxel_at(const ColliderSet& cs, const DCollider& c, int32_t x, int32_t y,
                                             int32_t z) {
    const int32_t bx = (x >> 3) - c.bmin[0], by = (y >> 3) - c.bmin[1], bz = (z >> 3) - c.bmin[2];
    if ((uint32_t)bx >= (uint32_t)c.bdim[0] || (uint32_t)by >= (uint32_t)c.bdim[1] ||
        (uint32_t)bz >= (uint32_t)c.bdim[2])
        return 0u;
    const int32_t slot = __ldg(&cs.grid[c.grid_off + (uint32_t)(bx + c.bdim[0] * (by + c.bdim[1] * bz))]);
    if (slot < 0) return 0u;
    return (uint32_t)__ldg(&cs.vox[(size_t)(c.brick_off + (uint32_t)slot) * 512u + (uint32_t)((x & 7) + 8 * (y & 7) +
                                                                                                 64 * (z & 7))]);
}
// The masks of table entry e (the probe centre at offset e of [min_bound - 1,
// max_bound], x fastest, extents ex, ey): the same 27 lookups and clipping as
// a probe.
__device__ __forceinline__ uint4 nbhd_entry(const ColliderSet& cs, const DCollider& c, uint32_t e, uint32_t ex,
                                            uint32_t ey) {
    const int32_t x = c.min_bound[0] - 1 + (int32_t)(e % ex), y = c.min_bound[1] - 1 + (int32_t)((e / ex) % ey),
                  z = c.min_bound[2] - 1 + (int32_t)(e / (ex * ey));
    uint32_t ne = 0u, co = 0u, ec = 0u, in = 0u;
    for (uint32_t k = 0; k < 27u; ++k) {
        const int32_t bx = x + (int32_t)(k % 3u) - 1, by = y + (int32_t)((k / 3u) % 3u) - 1,
                      bz = z + (int32_t)(k / 9u) - 1;
        if (bx < c.min_bound[0] || bx >= c.max_bound[0] || by < c.min_bound[1] || by >= c.max_bound[1] ||
            bz < c.min_bound[2] || bz >= c.max_bound[2])
            continue;
        const uint32_t tb = vtype(voxel_at(cs, c, bx, by, bz));
        ne |= (uint32_t)(tb != kEmpty) << k;
        co |= (uint32_t)(tb == kCorner) << k;
        ec |= (uint32_t)(tb == kCorner || tb == kEdge) << k;
        in |= (uint32_t)(tb == kInside) << k;
    }
    return make_uint4(ne, co, ec, in);
}
// The neighbourhood masks of the listed colliders' probe centres
// (DCollider::nb_off; every collider when list is null): one thread per centre.
__global__ void k_nbhd_build(ColliderSet cs, uint4* nb, const uint32_t* list, uint32_t n_list) {
    const uint32_t n = list ? n_list : cs.n;
    for (uint32_t li = blockIdx.y; li < n; li += gridDim.y) {
        const DCollider& c = cs.c[list ? list[li] : li];
        if (c.nb_off == kNoTable) continue;
        const uint32_t ex = (uint32_t)(c.max_bound[0] - c.min_bound[0]) + 2u,
                       ey = (uint32_t)(c.max_bound[1] - c.min_bound[1]) + 2u,
                       ez = (uint32_t)(c.max_bound[2] - c.min_bound[2]) + 2u;
        const uint32_t total = ex * ey * ez;
        for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x)
            nb[c.nb_off + e] = nbhd_entry(cs, c, e, ex, ey);
    }
}
// Slot of the brick at brick coordinates (bx, by, bz), or -1.
__device__ __forceinline__ int32_t brick_slot(const ColliderSet& cs, const DCollider& c, int32_t bx, int32_t by,
                                              int32_t bz) {
    bx -= c.bmin[0];
    by -= c.bmin[1];
    bz -= c.bmin[2];
    if ((uint32_t)bx >= (uint32_t)c.bdim[0] || (uint32_t)by >= (uint32_t)c.bdim[1] ||
        (uint32_t)bz >= (uint32_t)c.bdim[2])
        return -1;
    return __ldg(&cs.grid[c.grid_off + (uint32_t)(bx + c.bdim[0] * (by + c.bdim[1] * bz))]);
}
// Bricks holding voxels inside the inclusive voxel box [lo, hi], counted by
// the lanes of a warp (result in every lane).
__device__ uint32_t warp_count_bricks(const ColliderSet& cs, const DCollider& c, I3 lo, I3 hi) {
    const int32_t x0 = lo.x >> 3, y0 = lo.y >> 3, z0 = lo.z >> 3;
    const int32_t nx = (hi.x >> 3) - x0 + 1, ny = (hi.y >> 3) - y0 + 1, nz = (hi.z >> 3) - z0 + 1;
    uint32_t cnt = 0;
    if (nx > 0 && ny > 0 && nz > 0) {
        const uint32_t cells = (uint32_t)(nx * ny * nz);
        for (uint32_t i = threadIdx.x & 31; i < cells; i += 32u) {
            const int32_t bx = x0 + (int32_t)(i % (uint32_t)nx), by = y0 + (int32_t)((i / (uint32_t)nx) % (uint32_t)ny),
                          bz = z0 + (int32_t)(i / ((uint32_t)nx * (uint32_t)ny));
            if (brick_slot(cs, c, bx, by, bz) >= 0) ++cnt;
        }
    }
    return warp_sum(cnt);
}

__device__ __forceinline__ F3 voxel_to_local(float vs, int32_t x, int32_t y, int32_t z) {
    const float half = vs * 0.5f;
    return F3{(float)x * vs + half, (float)y * vs + half, (float)z * vs + half};
}
__device__ __forceinline__ I3 local_to_voxel(float vs, F3 p) {
    return I3{(int32_t)floorf(p.x / vs), (int32_t)floorf(p.y / vs), (int32_t)floorf(p.z / vs)};
}
__device__ __forceinline__ bool valid_coord(const DCollider& c, int32_t x, int32_t y, int32_t z) {
    return x >= c.min_bound[0] && x < c.max_bound[0] && y >= c.min_bound[1] && y < c.max_bound[1] &&
           z >= c.min_bound[2] && z < c.max_bound[2];
}

// NORMAL_LUT (collision_voxel.zig:47-76) as getNormalVec3 would return it.
__device__ __forceinline__ F3 lut_normal(uint32_t idx) {
    if (idx >= 26u) return F3{0.f, 0.f, 0.f};
    // component codes: 0 -> 0, 1 -> +1, 2 -> -1, packed 2 bits per axis
    const uint32_t kCode[26] = {0x01, 0x02, 0x04, 0x08, 0x10, 0x20, 0x05, 0x09, 0x06, 0x0A, 0x11, 0x21, 0x12,
                                0x22, 0x14, 0x24, 0x18, 0x28, 0x15, 0x25, 0x19, 0x29, 0x16, 0x26, 0x1A, 0x2A};
    const uint32_t c = kCode[idx];
    const float x = (c & 3u) == 1u ? 1.f : ((c & 3u) == 2u ? -1.f : 0.f);
    const float y = ((c >> 2) & 3u) == 1u ? 1.f : (((c >> 2) & 3u) == 2u ? -1.f : 0.f);
    const float z = ((c >> 4) & 3u) == 1u ? 1.f : (((c >> 4) & 3u) == 2u ? -1.f : 0.f);
    return normalize3(F3{x, y, z});
}

// ---------------------------------------------------------------------------
// OBB helpers (math.zig:715-747) and SAT (narrow_phase.zig:505-569)
// ---------------------------------------------------------------------------
struct Obb {
    F3 c, h;
    Qt q;
};
__device__ __forceinline__ Obb obb_from(const DCollider& col, F3 pos, Qt q) {
    const F3 mn{col.aabb_min[0], col.aabb_min[1], col.aabb_min[2]};
    const F3 mx{col.aabb_max[0], col.aabb_max[1], col.aabb_max[2]};
    const F3 center = (mn + mx) * 0.5f;
    const F3 ext = (mx - mn) * 0.5f;
    return Obb{transform_point(pos, q, center), ext, q};
}
__device__ __forceinline__ void obb_axes(const Obb& o, F3 ax[3]) {
    ax[0] = qrotate(o.q, F3{1.f, 0.f, 0.f});
    ax[1] = qrotate(o.q, F3{0.f, 1.f, 0.f});
    ax[2] = qrotate(o.q, F3{0.f, 0.f, 1.f});
}
__device__ __forceinline__ void obb_verts(const Obb& o, F3 v[8]) {
    F3 ax[3];
    obb_axes(o, ax);
    const F3 ex = ax[0] * o.h.x, ey = ax[1] * o.h.y, ez = ax[2] * o.h.z;
    v[0] = ((o.c - ex) - ey) - ez;
    v[1] = ((o.c + ex) - ey) - ez;
    v[2] = ((o.c - ex) + ey) - ez;
    v[3] = ((o.c + ex) + ey) - ez;
    v[4] = ((o.c - ex) - ey) + ez;
    v[5] = ((o.c + ex) - ey) + ez;
    v[6] = ((o.c - ex) + ey) + ez;
    v[7] = ((o.c + ex) + ey) + ez;
}
__device__ __forceinline__ void project8(const F3 v[8], F3 axis, float* mn, float* mx) {
    float lo = __int_as_float(0x7f800000), hi = -__int_as_float(0x7f800000);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const float p = dot3(v[i], axis);
        lo = fminf(lo, p);
        hi = fmaxf(hi, p);
    }
    *mn = lo;
    *mx = hi;
}
__device__ bool sat_separated(const Obb& a, const Obb& b) {
    F3 aa[3], ab[3], va[8], vb[8];
    obb_axes(a, aa);
    obb_axes(b, ab);
    obb_verts(a, va);
    obb_verts(b, vb);
    float p0, p1, q0, q1;
    for (int i = 0; i < 3; ++i) {
        project8(va, aa[i], &p0, &p1);
        project8(vb, aa[i], &q0, &q1);
        if (p1 < q0 || q1 < p0) return true;
    }
    for (int i = 0; i < 3; ++i) {
        project8(va, ab[i], &p0, &p1);
        project8(vb, ab[i], &q0, &q1);
        if (p1 < q0 || q1 < p0) return true;
    }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            const F3 cr = cross3(aa[i], ab[j]);
            const float l = len3(cr);
            if (l < 0.001f) continue;
            const F3 ax = cr * (1.0f / l);
            project8(va, ax, &p0, &p1);
            project8(vb, ax, &q0, &q1);
            if (p1 < q0 || q1 < p0) return true;
        }
    return false;
}

// getOverlapRegion (narrow_phase.zig:644-698).  Returns false when empty.
__device__ bool overlap_region(const DCollider& ca, F3 pa, Qt qa, const DCollider& cb, F3 pb, Qt qb, I3* rmin,
                               I3* rmax) {
    const Obb ob = obb_from(cb, pb, qb);
    F3 vb[8];
    obb_verts(ob, vb);
    const Qt inv = qconj(qa);
    const float inf = __int_as_float(0x7f800000);
    F3 tmn{inf, inf, inf}, tmx{-inf, -inf, -inf};
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const F3 rel = qrotate(inv, vb[i] - pa);
        tmn = min3(tmn, rel);
        tmx = max3(tmx, rel);
    }
    const float vs = ca.vs;
    tmn = tmn - F3{vs, vs, vs};
    tmx = tmx + F3{vs, vs, vs};
    const F3 lo{ca.aabb_min[0], ca.aabb_min[1], ca.aabb_min[2]};
    const F3 hi{ca.aabb_max[0], ca.aabb_max[1], ca.aabb_max[2]};
    const F3 mnc = clamp3(tmn, lo, hi), mxc = clamp3(tmx, lo, hi);
    if (mnc.x >= mxc.x || mnc.y >= mxc.y || mnc.z >= mxc.z) return false;
    const I3 a = local_to_voxel(vs, mnc), b = local_to_voxel(vs, mxc);
    *rmin = I3{max(a.x, ca.min_bound[0]), max(a.y, ca.min_bound[1]), max(a.z, ca.min_bound[2])};
    *rmax = I3{min(b.x, ca.max_bound[0]), min(b.y, ca.max_bound[1]), min(b.z, ca.max_bound[2])};
    return true;
}

// BrickPairKey.hash with zero brick positions, and computeTransformHash
// (narrow_phase.zig:118-169).
__device__ __forceinline__ unsigned long long cache_transform_hash(F3 rp, Qt rr) {
    const int32_t qx = (int32_t)(rp.x * 100.0f), qy = (int32_t)(rp.y * 100.0f), qz = (int32_t)(rp.z * 100.0f);
    const int16_t rw = (int16_t)(int32_t)clampf_ref(rr.w * 1000.0f, -32767.0f, 32767.0f);
    const int16_t rx = (int16_t)(int32_t)clampf_ref(rr.x * 1000.0f, -32767.0f, 32767.0f);
    const int16_t ry = (int16_t)(int32_t)clampf_ref(rr.y * 1000.0f, -32767.0f, 32767.0f);
    const int16_t rz = (int16_t)(int32_t)clampf_ref(rr.z * 1000.0f, -32767.0f, 32767.0f);
    unsigned long long h = 0;
    h = h * 31ull + (unsigned long long)(uint32_t)qx;
    h = h * 31ull + (unsigned long long)(uint32_t)qy;
    h = h * 31ull + (unsigned long long)(uint32_t)qz;
    h = h * 31ull + (unsigned long long)(uint16_t)rw;
    h = h * 31ull + (unsigned long long)(uint16_t)rx;
    h = h * 31ull + (unsigned long long)(uint16_t)ry;
    h = h * 31ull + (unsigned long long)(uint16_t)rz;
    return h;
}
__device__ __forceinline__ unsigned long long cache_key_hash(uint32_t a, uint32_t b, unsigned long long th) {
    unsigned long long h = 0;
    h = h * 31ull + (unsigned long long)a;
    h = h * 31ull + (unsigned long long)b;
#pragma unroll
    for (int i = 0; i < 6; ++i) h = h * 31ull;  // brick positions (0,0,0), (0,0,0)
    h = h * 31ull + th;
    return h;
}

// Hash table of pair keys (open addressing).
__device__ __forceinline__ uint32_t ht_hash(unsigned long long k, uint32_t cap) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ull;
    k ^= k >> 33;
    return (uint32_t)k & (cap - 1u);
}
__device__ void ht_insert(HashSlot* t, uint32_t cap, unsigned long long key, uint32_t idx) {
    uint32_t s = ht_hash(key, cap);
    for (uint32_t i = 0; i < cap; ++i) {
        const unsigned long long prev = atomicCAS(&t[s].key, 0ull, key);
        if (prev == 0ull || prev == key) {
            t[s].idx = idx;
            return;
        }
        s = (s + 1u) & (cap - 1u);
    }
}
__device__ uint32_t ht_find(const HashSlot* t, uint32_t cap, unsigned long long key) {
    uint32_t s = ht_hash(key, cap);
    for (uint32_t i = 0; i < cap; ++i) {
        const unsigned long long k = t[s].key;
        if (k == key) return t[s].idx;
        if (k == 0ull) return 0xFFFFFFFFu;
        s = (s + 1u) & (cap - 1u);
    }
    return 0xFFFFFFFFu;
}

__device__ __forceinline__ uint32_t find_body(const uint2* ids, uint32_t n, uint32_t id) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        const uint32_t v = ids[mid].x;
        if (v < id) lo = mid + 1;
        else hi = mid;
    }
    return (lo < n && ids[lo].x == id) ? ids[lo].y : 0xFFFFFFFFu;
}

// ---------------------------------------------------------------------------
// Phase: begin (sleep skip test, per-body step-start state)
// ---------------------------------------------------------------------------
template <class G>
__device__ bool phase_begin(G& g, WorldDev& w, bool skip_test, bool* skipped) {
    // counters (not the sticky error word) are zeroed by the host/graph memset.
    for (uint32_t i = g.rank(); i < w.n_bodies; i += g.size()) {
        const DBodyProp& pr = w.prop[i];
        if (pr.type == 2u && !pr.sleeping) atomicAdd(&w.ctr[C_AWAKE], 1u);
    }
    if (!g.sync()) return false;
    const uint32_t awake = *(volatile uint32_t*)&w.ctr[C_AWAKE];
    // VoxelPhysicsSystem.step returns early when every dynamic body sleeps
    // (system.zig:538-544)
    if (skip_test && w.cfg.sleeping_on && awake == 0u) {
        *skipped = true;
        if (g.rank() == 0) w.ctr[C_STEP_SKIPPED] = 1u;
        return true;
    }
    *skipped = false;
    // BodyState.fromBody: world inverse inertia from the current rotation.
    for (uint32_t i = g.rank(); i < w.n_bodies; i += g.size()) {
        DBody& b = w.body[i];
        const DBodyProp& pr = w.prop[i];
        const Qt q = qof(b.q);
        w.qn[i] = f4of(qnormalize(q));
        w.p0[i] = b.p;
        if (b.p.w == 0.0f) {
            b.i0 = b.i1 = b.i2 = make_float4(0.f, 0.f, 0.f, 0.f);
        } else {
            M33 il;
#pragma unroll
            for (int k = 0; k < 9; ++k) il.m[k] = pr.il[k];
            const M33 m = world_inv_inertia(q, il);
            b.i0 = make_float4(m.m[0], m.m[1], m.m[2], 0.f);
            b.i1 = make_float4(m.m[3], m.m[4], m.m[5], 0.f);
            b.i2 = make_float4(m.m[6], m.m[7], m.m[8], 0.f);
        }
    }
    return g.sync();
}

// ---------------------------------------------------------------------------
// Phase: broad phase (the pair list of the step, built on the device)
// ---------------------------------------------------------------------------
// The reference hands narrowPhase() the pairs of its AABB trees
// (broad_phase.zig:606-619).  This pair source keeps every (min id, max id)
// pair, not both static, whose world AABBs (AABB.transform of the collider's
// local AABB, math.zig:686-693) inflated by `margin` overlap, sorted by
// (body_a, body_b): one warp per id-sorted row, lanes sweeping the later
// rows, a ballot keeping them in order.  The sweep counts each row's pairs;
// after a scan of the counts the pairs are written from the hit masks the
// sweep kept (worlds with mask room), else by sweeping again.  *overflow:
// the list does not fit pair_cap (nothing is written; the host grows the
// buffers).
template <class G>
__device__ bool phase_broadphase(G& g, WorldDev& w, const ColliderSet& cs, bool* overflow, unsigned char* smem) {
    const uint32_t N = w.n_bodies;
    const float m = w.cfg.margin;
    // inflated world AABBs in id order (position s holds body ids[s]), w = 1
    // for a static body, so that the sweep below reads them coalesced
    for (uint32_t s = g.rank(); s < N; s += g.size()) {
        const uint32_t i = w.ids[s].y;
        const DBody b = w.body[i];
        const F3 x = f3of(b.p);
        const Qt q = qof(b.q);
        F3 lo, hi;
        const uint32_t ci = w.prop[i].collider;
        if (ci < cs.n) {
            const DCollider& c = cs.c[ci];
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
        lo = lo - F3{m, m, m};
        hi = hi + F3{m, m, m};
        w.aabb_mn[s] = make_float4(lo.x, lo.y, lo.z, w.prop[i].type == 0u ? 1.f : 0.f);
        w.aabb_mx[s] = make_float4(hi.x, hi.y, hi.z, 0.f);
    }
    if (!g.sync()) return false;
    const uint32_t lane = threadIdx.x & 31, wid = g.rank() >> 5, nw = g.size() >> 5;
    const bool masks = w.bpmask != nullptr && N <= w.bp_rows;
    if (g.rank() == 0 && w.ts) w.ts[TS_BP_AABB] = global_ns();
    // The count pass with the boxes staged in shared memory, kBpTile at a
    // time, when every warp holds at most one row pair and the hit masks are
    // kept (the grid launch): each warp tests the 32-column chunks of its two
    // rows that start in the tile (the tile holds 32 boxes more for the
    // chunks that run past its end).  The same chunks, masks and counts as
    // the sweep below; its write pass follows.
    // tiles of up to 512 boxes, as many as the launch's dynamic shared memory
    // holds (each tile is one round trip to L2 for the block)
    uint32_t dyn = 0;
    asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
    const uint32_t kBpTile = min(512u, (dyn / (2u * (uint32_t)sizeof(float4)) > 32u
                                            ? dyn / (2u * (uint32_t)sizeof(float4)) - 32u
                                            : 0u) & ~31u);
    const uint32_t kBpSpan = kBpTile + 32u;
    const bool tiled = masks && smem != nullptr && (N + 1u) / 2u <= nw && kBpTile >= 128u;
    if (tiled) {
        float4* tmn = reinterpret_cast<float4*>(smem);
        float4* tmx = tmn + kBpSpan;
        const uint32_t r = wid;
        const bool rows = r < (N + 1u) / 2u;
        const uint32_t s2[2] = {r, N - 1u - r};
        bool act[2], si[2];
        float4 a0[2], a1[2];
        uint32_t cnt[2] = {0u, 0u};
#pragma unroll
        for (uint32_t h = 0; h < 2u; ++h) {
            act[h] = rows && !(h && s2[1] == r);
            a0[h] = act[h] ? w.aabb_mn[s2[h]] : make_float4(0.f, 0.f, 0.f, 0.f);
            a1[h] = act[h] ? w.aabb_mx[s2[h]] : make_float4(0.f, 0.f, 0.f, 0.f);
            si[h] = a0[h].w != 0.f;
        }
        for (uint32_t tile0 = 0; tile0 < N; tile0 += kBpTile) {
            __syncthreads();
            for (uint32_t x = threadIdx.x; x < kBpSpan; x += blockDim.x) {
                const uint32_t t = tile0 + x;
                if (t < N) {
                    tmn[x] = w.aabb_mn[t];
                    tmx[x] = w.aabb_mx[t];
                }
            }
            __syncthreads();
#pragma unroll
            for (uint32_t h = 0; h < 2u; ++h) {
                if (!act[h]) continue;
                const uint32_t s = s2[h];
                // this row's chunks c = s + 1 + 32 j that start in the tile
                uint32_t c = s + 1u;
                if (c < tile0) c += (tile0 - c + 31u) / 32u * 32u;
                for (; c < tile0 + kBpTile && c < N; c += 32u) {
                    const uint32_t t = c + lane;
                    bool hit = false;
                    if (t < N) {
                        const float4 b0 = tmn[t - tile0], b1 = tmx[t - tile0];
                        hit = !(si[h] && b0.w != 0.f) && a0[h].x <= b1.x && a1[h].x >= b0.x && a0[h].y <= b1.y &&
                              a1[h].y >= b0.y && a0[h].z <= b1.z && a1[h].z >= b0.z;
                    }
                    const uint32_t mk = __ballot_sync(0xffffffffu, hit);
                    if (lane == 0) w.bpmask[(size_t)s * w.bp_stride + (c - s - 1u) / 32u] = mk;
                    cnt[h] += (uint32_t)__popc(mk);
                }
            }
        }
        if (lane == 0) {
            if (act[0]) w.pcount[s2[0]] = cnt[0];
            if (act[1]) w.pcount[s2[1]] = cnt[1];
        }
        if (!g.sync()) return false;
    }
    for (int pass = tiled ? 1 : 0; pass < 2; ++pass) {
        if (pass == 1) {
            if (g.rank() == 0 && w.ts) w.ts[TS_BP_COUNT] = global_ns();
            uint32_t total = 0;
            if (!group_scan(
                    g, N, [&](uint32_t i) { return w.pcount[i]; }, [&](uint32_t i, uint32_t pre) { w.poff[i] = pre; },
                    w.scan, &total))
                return false;
            if (g.rank() == 0 && w.ts) w.ts[TS_BP_SCAN] = global_ns();
            *overflow = total > w.pair_cap;
            w.n_pairs = total;
            if (g.rank() == 0) *w.n_pairs_dev = total;
            if (*overflow) return true;
        }
        // a warp takes rows r and N - 1 - r (about N columns in all)
        for (uint32_t r = wid; r < (N + 1u) / 2u; r += nw) {
            for (uint32_t h = 0; h < 2u; ++h) {
                const uint32_t s = h ? N - 1u - r : r;
                if (h && s == r) break;
                if (pass && masks) {
                    // the row's pairs from its masks, 32 mask words at a time
                    const uint32_t nj = (N - 1u - s + 31u) / 32u;
                    const uint32_t* mrow = w.bpmask + (size_t)s * w.bp_stride;
                    uint32_t o = w.poff[s];
                    const uint32_t ida = w.ids[s].x;
                    for (uint32_t jb = 0; jb < nj; jb += 32u) {
                        const uint32_t j = jb + lane;
                        uint32_t mk = j < nj ? mrow[j] : 0u;
                        const uint32_t c = (uint32_t)__popc(mk);
                        const uint32_t inc = warp_incl_scan(c);
                        uint32_t q = o + inc - c;
                        for (; mk; mk &= mk - 1u)
                            w.pairs[q++] = make_uint2(ida, w.ids[s + 1u + 32u * j + (uint32_t)(__ffs(mk) - 1)].x);
                        o += __shfl_sync(0xffffffffu, inc, 31);
                    }
                    continue;
                }
                const float4 a0 = w.aabb_mn[s], a1 = w.aabb_mx[s];
                const bool si = a0.w != 0.f;
                uint32_t o = pass ? w.poff[s] : 0u;
                uint32_t cnt = 0;
                auto test = [&](uint32_t t) {
                    bool hit = false;
                    if (t < N) {
                        const float4 b0 = __ldg(w.aabb_mn + t), b1 = __ldg(w.aabb_mx + t);
                        hit = !(si && b0.w != 0.f) && a0.x <= b1.x && a1.x >= b0.x && a0.y <= b1.y &&
                              a1.y >= b0.y && a0.z <= b1.z && a1.z >= b0.z;
                    }
                    return hit;
                };
                auto emit = [&](bool hit, uint32_t t) {
                    const uint32_t mk = __ballot_sync(0xffffffffu, hit);
                    if (masks && lane == 0) w.bpmask[(size_t)s * w.bp_stride + (t - lane - s - 1u) / 32u] = mk;
                    if (pass && hit)
                        w.pairs[o + __popc(mk & ((1u << lane) - 1u))] = make_uint2(w.ids[s].x, w.ids[t].x);
                    o += __popc(mk);
                    cnt += __popc(mk);
                };
                // four chunks of 32 columns per iteration, all tested before
                // any is counted
                for (uint32_t t0 = s + 1; t0 < N; t0 += 128u) {
                    const bool h0 = test(t0 + lane), h1 = test(t0 + 32u + lane), h2 = test(t0 + 64u + lane),
                               h3 = test(t0 + 96u + lane);
                    emit(h0, t0 + lane);
                    if (t0 + 32u < N) emit(h1, t0 + 32u + lane);
                    if (t0 + 64u < N) emit(h2, t0 + 64u + lane);
                    if (t0 + 96u < N) emit(h3, t0 + 96u + lane);
                }
                if (!pass && lane == 0) w.pcount[s] = cnt;
            }
        }
        if (!g.sync()) return false;
    }
    return true;
}

// ---------------------------------------------------------------------------
// Phase: pairs (system.narrowPhase filter + processPair head)
// ---------------------------------------------------------------------------
template <class G>
__device__ bool phase_pairs(G& g, WorldDev& w, const ColliderSet& cs, uint32_t cur) {
    const uint32_t P = w.n_pairs;
    if (g.rank() == 0) {
        w.ctr[C_PAIRS_IN] = P;
        w.cframe[0] += 1ull;  // BrickPairCache.beginFrame
    }
    for (uint32_t i = g.rank(); i < w.ht_cap; i += g.size()) {
        w.ht[cur][i].key = 0ull;
        w.ht[cur][i].idx = 0xFFFFFFFFu;
    }
    for (uint32_t p = g.rank(); p < P; p += g.size()) {
        const uint2 pr = w.pairs[p];
        const uint32_t ia = find_body(w.ids, w.n_bodies, pr.x), ib = find_body(w.ids, w.n_bodies, pr.y);
        uint32_t fl = 0;
        if (ia == 0xFFFFFFFFu || ib == 0xFFFFFFFFu) fl |= PF_INVALID;
        const bool as = ia != 0xFFFFFFFFu ? w.prop[ia].sleeping != 0u : false;
        const bool bs = ib != 0xFFFFFFFFu ? w.prop[ib].sleeping != 0u : false;
        if (as && bs) fl |= PF_CARRY;
        PairInfo& pi = w.pinfo[p];
        pi.ia = ia;
        pi.ib = ib;
        pi.flags = fl;
        pi.voxels_checked = 0;
        pi.candidates = 0;
        pi.hit = 0u;
        pi.cache_slot = 0xFFFFFFFFu;
        w.flag[p] = (fl & PF_CARRY) ? 0u : 1u;
    }
    if (!g.sync()) return false;
    if (g.rank() == 0 && w.ts) w.ts[TS_PR_IDS] = global_ns();
    if (w.cfg.reference_caps) {
        uint32_t tot;
        if (!group_scan(
                g, P, [&](uint32_t i) { return w.flag[i]; },
                [&](uint32_t i, uint32_t pre) {
                    if (w.flag[i] && pre >= 512u) w.pinfo[i].flags |= PF_DROPPED;
                },
                w.scan, &tot))
            return false;
    }
    uint32_t tested = 0;
    for (uint32_t p = g.rank(); p < P; p += g.size()) {
        PairInfo& pi = w.pinfo[p];
        uint32_t fl = pi.flags;
        if (fl & (PF_CARRY | PF_DROPPED | PF_INVALID)) continue;
        fl |= PF_TESTED;
        ++tested;
        const DBody& A = w.body[pi.ia];
        const DBody& B = w.body[pi.ib];
        const DBodyProp& pa = w.prop[pi.ia];
        const DBodyProp& pb = w.prop[pi.ib];
        if (pa.collider >= cs.n || pb.collider >= cs.n) {
            pi.flags = fl | PF_NOCOLL;
            continue;
        }
        const DCollider& ca = cs.c[pa.collider];
        const DCollider& cb = cs.c[pb.collider];
        const F3 xa = f3of(A.p), xb = f3of(B.p);
        const Qt qa = qof(A.q), qb = qof(B.q);
        if (w.cfg.use_sat) {
            if (sat_separated(obb_from(ca, xa, qa), obb_from(cb, xb, qb))) {
                pi.flags = fl | PF_SEPARATED;
                continue;
            }
        }
        const bool use_cache =
            w.cfg.use_cache && (pa.type == 0u || pb.type == 0u || pa.sleeping != 0u || pb.sleeping != 0u);
        if (use_cache) {
            fl |= PF_CACHE;
            const F3 rp = xb - xa;
            const Qt rr = qmul(qconj(qa), qb);
            const bool af = pa.id < pb.id;
            pi.key_a = af ? pa.id : pb.id;
            pi.key_b = af ? pb.id : pa.id;
            pi.th = cache_transform_hash(rp, rr);
        } else {
            fl |= PF_DETECT;
        }
        I3 rmin, rmax;
        if (overlap_region(ca, xa, qa, cb, xb, qb, &rmin, &rmax)) {
            if (rmin.x <= rmax.x && rmin.y <= rmax.y && rmin.z <= rmax.z) {
                fl |= PF_REGION;
                // a large region is probed by a whole CTA (listed in w.cons,
                // which is free until phase_constraints)
                const unsigned long long V = (unsigned long long)(rmax.x - rmin.x + 1) *
                                             (unsigned long long)(rmax.y - rmin.y + 1) *
                                             (unsigned long long)(rmax.z - rmin.z + 1);
                if (w.cfg.heavy_voxels && V >= w.cfg.heavy_voxels) {
                    fl |= PF_HEAVY;
                    w.cons[atomicAdd(&w.ctr[C_NHEAVY], 1u)] = p;
                }
            }
            pi.rmin[0] = rmin.x; pi.rmin[1] = rmin.y; pi.rmin[2] = rmin.z;
            pi.rmax[0] = rmax.x; pi.rmax[1] = rmax.y; pi.rmax[2] = rmax.z;
        }
        pi.flags = fl;
    }
    tested = warp_sum(tested);
    if ((threadIdx.x & 31) == 0 && tested) atomicAdd(&w.ctr[C_PAIRS_TESTED], tested);
    if (!g.sync()) return false;
    if (g.rank() == 0 && w.ts) w.ts[TS_PR_SAT] = global_ns();
    if (w.cfg.use_cache) {
        // the lookups of the pairs consulting the cache, in pair order, for
        // the replay warp (window starts computed here, off its chain)
        uint32_t nc = 0;
        if (!group_scan(
                g, P, [&](uint32_t i) { return (w.pinfo[i].flags & PF_CACHE) ? 1u : 0u; },
                [&](uint32_t i, uint32_t pre) {
                    const PairInfo& pi = w.pinfo[i];
                    if (pi.flags & PF_CACHE) {
                        CacheLook r;
                        r.p = i;
                        r.a = pi.key_a;
                        r.b = pi.key_b;
                        r.th = pi.th;
                        r.start = (uint32_t)(cache_key_hash(r.a, r.b, r.th) % (unsigned long long)w.cache_cap);
                        w.clist[pre] = r;
                    }
                },
                w.scan, &nc))
            return false;
        if (g.rank() == 0) w.ctr[C_NCACHE] = nc;
        return g.sync();
    }
    return true;
}

// ---------------------------------------------------------------------------
// Brick-pair cache replay (BrickPairCache.get / put, narrow_phase.zig:228-302)
// ---------------------------------------------------------------------------
// The hit / miss decision of every cache lookup depends only on the keys and
// on the order of the lookups, not on any contact value: a lookup is a get
// (probe at most 16 slots from hash % capacity: stop at an empty slot = miss
// or at the key = hit, which refreshes last_used) and, after a miss, a put
// (the first empty slot of the window, else evict its least recently used
// entry).  One warp replays the keys of this step in pair order on a
// shared-memory copy of the table while the other warps already detect every
// cache-consulting pair; a hit later discards that detection and replays the
// cached contacts instead.  Values are written after detection
// (phase_finalize), the last writer of a slot winning, as the sequential puts
// would leave them.
//
// A lookup reads and writes only its window, so it sees the state the
// sequential replay gives it once every earlier lookup whose window overlaps
// its own has run.  The warp keeps up to 32 pending lookups in order, one per
// lane; each round every pending lookup whose window overlaps no earlier
// pending one runs (their windows are disjoint), the rest move up in order
// and new ones fill the free lanes.  Keys stream in 32 at a time, one batch
// ahead.

// Position of the n-th (from 0) set bit of m; n < popc(m).
__device__ __forceinline__ uint32_t nth_set_bit(uint32_t m, uint32_t n) {
    uint32_t r = 0;
#pragma unroll
    for (uint32_t wd = 16; wd; wd >>= 1) {
        const uint32_t c = (uint32_t)__popc(m & ((1u << wd) - 1u));
        if (n >= c) {
            n -= c;
            m >>= wd;
            r += wd;
        }
    }
    return r;
}

__device__ void cache_replay(WorldDev& w, const CacheSmem& t) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t cap = w.cache_cap;
    const uint32_t maxp = cap < 16u ? cap : 16u;
    const uint32_t frame = (uint32_t)w.cframe[0];
    const uint32_t n = w.ctr[C_NCACHE];
    for (uint32_t i = lane; i < cap; i += 32u) {
        const CacheKeyRec k = w.ckey[i];
        t.ab[i] = make_uint2(k.a, k.b);
        t.th[i] = k.th;
        t.lu[i] = k.valid ? (uint32_t)k.last_used : 0u;
    }
    __syncwarp();
    uint32_t hits = 0, misses = 0, evictions = 0;
    // the lookups stream into this SM's L1 ahead of use (nothing else runs
    // here): their 128-byte lines, all requests in flight at once
    {
        const char* base = reinterpret_cast<const char*>(w.clist);
        const uint32_t lines = (uint32_t)(((size_t)n * sizeof(CacheLook) + 127u) / 128u);
        for (uint32_t i = lane; i < lines; i += 32u)
            asm volatile("prefetch.global.L1 [%0];" ::"l"(base + (size_t)i * 128u));
    }
    using Look = CacheLook;
    auto load = [&](uint32_t idx) {
        Look r{0u, 0u, 0u, 0u, 0ull};
        if (idx < n) r = w.clist[idx];
        return r;
    };
    auto shfl = [&](const Look& x, uint32_t src) {
        Look r;
        r.p = __shfl_sync(0xffffffffu, x.p, src);
        r.a = __shfl_sync(0xffffffffu, x.a, src);
        r.b = __shfl_sync(0xffffffffu, x.b, src);
        r.start = __shfl_sync(0xffffffffu, x.start, src);
        r.th = __shfl_sync(0xffffffffu, x.th, src);
        return r;
    };
    // the windows starting at s0 and s1 (maxp slots each, mod cap) overlap
    auto overlap = [&](uint32_t s0, uint32_t s1) {
        const uint32_t d = s1 >= s0 ? s1 - s0 : s1 + cap - s0;
        return d < maxp || cap - d < maxp;
    };
    const bool coarse = cap >= 64u * maxp;
    Look cur = load(lane), nxt = load(32u + lane);  // keys [cb, cb + 32) and the batch after
    uint32_t cb = 0, taken = 0, np = 0;
    Look mine{0u, 0u, 0u, 0u, 0ull};
    for (;;) {
        // fill lanes np.. with the next keys, in order
        const uint32_t take = min(32u - np, n - taken);
        {
            const bool fill = lane >= np && lane < np + take;
            const uint32_t rc = fill ? taken + (lane - np) - cb : 0u;  // relative to cb, < 64
            const Look fc = shfl(cur, rc < 32u ? rc : 0u), fn = shfl(nxt, rc >= 32u ? rc - 32u : 0u);
            if (fill) mine = rc < 32u ? fc : fn;
        }
        taken += take;
        np += take;
        if (np == 0u) break;
        while (taken >= cb + 32u && cb + 32u < n) {
            cur = nxt;
            cb += 32u;
            nxt = load(cb + 32u + lane);
        }
        // ready: no earlier pending window overlaps this one.  With at least
        // 64 x maxp slots, overlapping windows start in the same or adjacent
        // sixty-fourths of the table, which a prefix OR over the lanes checks
        // (a conservative test); else every earlier window is compared.
        const bool pending = lane < np;
        bool ready = pending;
        if (coarse) {
            const uint32_t bk = (uint32_t)(((unsigned long long)mine.start * 64ull) / cap);
            const unsigned long long m = pending ? 1ull << bk : 0ull;
            unsigned long long inc = m;
#pragma unroll
            for (uint32_t d = 1; d < 32u; d <<= 1) {
                const unsigned long long o = __shfl_up_sync(0xffffffffu, inc, d);
                if (lane >= d) inc |= o;
            }
            unsigned long long ex = __shfl_up_sync(0xffffffffu, inc, 1);
            if (lane == 0u) ex = 0ull;
            const unsigned long long near = m | (m << 1) | (m >> 1) | (bk == 0u ? 1ull << 63 : 0ull) |
                                            (bk == 63u ? 1ull : 0ull);
            if (ex & near) ready = false;
        } else {
            for (uint32_t i = 0; i + 1u < np; ++i) {
                const uint32_t si = __shfl_sync(0xffffffffu, mine.start, i);
                if (i < lane && overlap(si, mine.start)) ready = false;
            }
        }
        if (ready) {
            // get: the first empty slot (miss) or the key (hit), whichever
            // comes first; put after a miss: that empty slot, else the first
            // least recently used one
            uint32_t fi = maxp, fm = maxp, mn = 0xFFFFFFFFu, mi = 0;
#pragma unroll
            for (uint32_t i = 0; i < 16u; ++i) {
                if (i >= maxp) break;
                uint32_t x = mine.start + i;
                if (x >= cap) x -= cap;
                const uint32_t lu = t.lu[x];
                const uint2 ab = t.ab[x];
                const unsigned long long th = t.th[x];
                if (lu == 0u) {
                    if (fi == maxp) fi = i;
                } else {
                    if (fm == maxp && ab.x == mine.a && ab.y == mine.b && th == mine.th) fm = i;
                    if (lu < mn) {
                        mn = lu;
                        mi = i;
                    }
                }
            }
            const bool hit = fm < fi;
            const bool evict = !hit && fi == maxp;
            uint32_t target = mine.start + (hit ? fm : (evict ? mi : fi));
            if (target >= cap) target -= cap;
            PairInfo& pi = w.pinfo[mine.p];
            t.lu[target] = frame;
            if (hit) {
                pi.hit = 1u;
                ++hits;
            } else {
                t.ab[target] = make_uint2(mine.a, mine.b);
                t.th[target] = mine.th;
                w.cwriter[target] = mine.p;
                pi.hit = 2u;
                ++misses;
                if (evict) ++evictions;
            }
            pi.cache_slot = target;
        }
        __syncwarp();
        // the lookups left move up, in order
        const uint32_t rm = __ballot_sync(0xffffffffu, pending && !ready);
        np = (uint32_t)__popc(rm);
        const Look moved = shfl(mine, lane < np ? nth_set_bit(rm, lane) : 0u);
        if (lane < np) mine = moved;
    }
    for (uint32_t i = lane; i < cap; i += 32u) {
        CacheKeyRec k;
        k.a = t.ab[i].x;
        k.b = t.ab[i].y;
        k.th = t.th[i];
        k.last_used = t.lu[i];
        k.valid = t.lu[i] != 0u ? 1u : 0u;
        k._pad = 0u;
        w.ckey[i] = k;
    }
    hits = warp_sum(hits);
    misses = warp_sum(misses);
    evictions = warp_sum(evictions);
    if (lane == 0) {
        w.ctr[C_CACHE_HITS] += hits;
        w.ctr[C_CACHE_MISSES] += misses;
        w.ctr[C_CACHE_EVICTIONS] += evictions;
        if (w.ts) w.ts[TS_CACHE] = global_ns();  // end of the replay (diagnostics)
    }
}

// The same replay on a whole CTA (the grid step's CTA 0, which detects
// nothing), for tables of at least 64 x 16 slots.  Up to kCtaReplayPending
// lookups are pending, in order, one per thread; each round every pending
// lookup whose window overlaps no earlier pending one is ready (the
// sixty-fourths prefix OR of cache_replay, over the block), the ready ones run
// at once, each scanned by sixteen lanes (a ballot finds the first empty slot
// and the key, a min-reduction the least recently used slot), and the rest
// move up in order.  The windows of a round are disjoint, so every lookup
// sees the state the sequential replay gives it.  scratch: at least
// cta_replay_scratch_bytes() bytes (the block's unused warp scratch).
constexpr uint32_t kCtaReplayPending = 256;
__host__ __device__ constexpr size_t cta_replay_scratch_bytes() {
    return 2u * kCtaReplayPending * sizeof(CacheLook) + kCtaReplayPending * sizeof(uint16_t) +
           32u * sizeof(unsigned long long) + 32u * sizeof(uint32_t) + 4u * sizeof(uint32_t);
}

__device__ void cache_replay_cta(WorldDev& w, const CacheSmem& t, unsigned char* scratch) {
    const uint32_t tid = threadIdx.x, T = blockDim.x, lane = tid & 31u, wid = tid >> 5;
    const uint32_t cap = w.cache_cap;
    const uint32_t frame = (uint32_t)w.cframe[0];
    const uint32_t n = w.ctr[C_NCACHE];
    CacheLook* bufA = reinterpret_cast<CacheLook*>(scratch);
    CacheLook* bufB = bufA + kCtaReplayPending;
    uint16_t* rdy = reinterpret_cast<uint16_t*>(bufB + kCtaReplayPending);
    unsigned long long* s_or = reinterpret_cast<unsigned long long*>(rdy + kCtaReplayPending);
    uint32_t* s_cnt = reinterpret_cast<uint32_t*>(s_or + 32);
    uint32_t* s_tot = s_cnt + 32;
    for (uint32_t i = tid; i < cap; i += T) {
        const CacheKeyRec k = w.ckey[i];
        t.ab[i] = make_uint2(k.a, k.b);
        t.th[i] = k.th;
        t.lu[i] = k.valid ? (uint32_t)k.last_used : 0u;
    }
    uint32_t hits = 0, misses = 0, evictions = 0;
    CacheLook* P = bufA;
    CacheLook* Q = bufB;
    uint32_t np = 0, taken = 0;
    const uint32_t nw = (kCtaReplayPending + 31u) / 32u;  // warps holding pending entries
    for (;;) {
        // fill the pending list up to its capacity, in order
        const uint32_t take = min(kCtaReplayPending - np, n - taken);
        for (uint32_t i = tid; i < take; i += T) P[np + i] = w.clist[taken + i];
        taken += take;
        np += take;
        __syncthreads();
        if (np == 0u) break;
        // ready: no earlier pending window in the same or an adjacent sixty-fourth
        const bool pending = tid < np;
        uint32_t bk = 0;
        unsigned long long m = 0ull;
        if (pending) {
            bk = (uint32_t)(((unsigned long long)P[tid].start * 64ull) / cap);
            m = 1ull << bk;
        }
        unsigned long long inc = m;
#pragma unroll
        for (uint32_t d = 1; d < 32u; d <<= 1) {
            const unsigned long long o = __shfl_up_sync(0xffffffffu, inc, d);
            if (lane >= d) inc |= o;
        }
        if (lane == 31u && wid < nw) s_or[wid] = inc;
        __syncthreads();
        unsigned long long ex = __shfl_up_sync(0xffffffffu, inc, 1);
        if (lane == 0u) ex = 0ull;
        for (uint32_t k = 0; k < wid && k < nw; ++k) ex |= s_or[k];
        const unsigned long long near =
            m | (m << 1) | (m >> 1) | (bk == 0u ? 1ull << 63 : 0ull) | (bk == 63u ? 1ull : 0ull);
        const bool ready = pending && !(ex & near);
        // positions: ready ones in a list, the others moved up into Q in order
        const uint32_t c = ready ? 1u : (pending ? 0x10000u : 0u);
        uint32_t ci = c;
#pragma unroll
        for (uint32_t d = 1; d < 32u; d <<= 1) {
            const uint32_t o = __shfl_up_sync(0xffffffffu, ci, d);
            if (lane >= d) ci += o;
        }
        if (lane == 31u && wid < nw) s_cnt[wid] = ci;
        __syncthreads();
        if (tid == 0) {
            uint32_t run = 0;
            for (uint32_t k = 0; k < nw; ++k) {
                const uint32_t v = s_cnt[k];
                s_cnt[k] = run;
                run += v;
            }
            *s_tot = run;
        }
        __syncthreads();
        const uint32_t off = (wid < nw ? s_cnt[wid] : 0u) + ci - c;
        if (ready) rdy[off & 0xFFFFu] = (uint16_t)tid;
        else if (pending) Q[off >> 16] = P[tid];
        __syncthreads();
        const uint32_t tot = *s_tot, nready = tot & 0xFFFFu;
        // the ready lookups, sixteen lanes each (the windows are disjoint)
        const uint32_t l16 = tid & 15u, grp = tid >> 4, ngrp = T >> 4;
        const uint32_t half = (lane >> 4) << 4;
        for (uint32_t j0 = 0; j0 < nready; j0 += ngrp) {
            const uint32_t j = j0 + grp;
            const bool act = j < nready;
            CacheLook L{0u, 0u, 0u, 0u, 0ull};
            if (act) L = P[rdy[j]];
            uint32_t x = L.start + l16;
            if (x >= cap) x -= cap;
            bool empty = false, match = false;
            unsigned long long key = ~0ull;
            if (act) {
                const uint32_t lu = t.lu[x];
                const uint2 ab = t.ab[x];
                const unsigned long long th = t.th[x];
                empty = lu == 0u;
                match = !empty && ab.x == L.a && ab.y == L.b && th == L.th;
                if (!empty) key = ((unsigned long long)lu << 32) | l16;
            }
            const uint32_t be = (__ballot_sync(0xffffffffu, empty) >> half) & 0xFFFFu;
            const uint32_t bm = (__ballot_sync(0xffffffffu, match) >> half) & 0xFFFFu;
#pragma unroll
            for (uint32_t d = 8; d > 0; d >>= 1) {
                const unsigned long long o = __shfl_xor_sync(0xffffffffu, key, d, 16);
                key = o < key ? o : key;
            }
            if (act && l16 == 0u) {
                const uint32_t fi = be ? (uint32_t)(__ffs(be) - 1) : 16u;
                const uint32_t fm = bm ? (uint32_t)(__ffs(bm) - 1) : 16u;
                const uint32_t mi = (uint32_t)(key & 0xFFFFu);
                const bool hit = fm < fi;
                const bool evict = !hit && fi == 16u;
                uint32_t target = L.start + (hit ? fm : (evict ? mi : fi));
                if (target >= cap) target -= cap;
                PairInfo& pi = w.pinfo[L.p];
                t.lu[target] = frame;
                if (hit) {
                    pi.hit = 1u;
                    ++hits;
                } else {
                    t.ab[target] = make_uint2(L.a, L.b);
                    t.th[target] = L.th;
                    w.cwriter[target] = L.p;
                    pi.hit = 2u;
                    ++misses;
                    if (evict) ++evictions;
                }
                pi.cache_slot = target;
            }
        }
        __syncthreads();
        CacheLook* tmp = P;
        P = Q;
        Q = tmp;
        np = tot >> 16;
    }
    for (uint32_t i = tid; i < cap; i += T) {
        CacheKeyRec k;
        k.a = t.ab[i].x;
        k.b = t.ab[i].y;
        k.th = t.th[i];
        k.last_used = t.lu[i];
        k.valid = t.lu[i] != 0u ? 1u : 0u;
        k._pad = 0u;
        w.ckey[i] = k;
    }
    hits = warp_sum(hits);
    misses = warp_sum(misses);
    evictions = warp_sum(evictions);
    if (lane == 0 && (hits | misses | evictions)) {
        atomicAdd(&w.ctr[C_CACHE_HITS], hits);
        atomicAdd(&w.ctr[C_CACHE_MISSES], misses);
        atomicAdd(&w.ctr[C_CACHE_EVICTIONS], evictions);
    }
    if (tid == 0 && w.ts) w.ts[TS_CACHE] = global_ns();  // end of the replay (diagnostics)
}

// ---------------------------------------------------------------------------
// Phase: probe (detectVoxelCollisions + checkNeighborhood + addContact)
// ---------------------------------------------------------------------------
// Top-4 multiset of penetrations, sorted descending, -inf padded.
struct Top4 {
    float v[4];
};
__device__ __forceinline__ Top4 top4_empty() {
    const float ni = -__int_as_float(0x7f800000);
    return Top4{{ni, ni, ni, ni}};
}
__device__ __forceinline__ void cswap_desc(float& a, float& b) {
    const float hi = fmaxf(a, b), lo = fminf(a, b);
    a = hi;
    b = lo;
}
// Top four of the union of two descending multisets.
__device__ __forceinline__ Top4 top4_merge(const Top4& a, const Top4& b) {
    Top4 c{{fmaxf(a.v[0], b.v[3]), fmaxf(a.v[1], b.v[2]), fmaxf(a.v[2], b.v[1]), fmaxf(a.v[3], b.v[0])}};
    cswap_desc(c.v[0], c.v[2]);
    cswap_desc(c.v[1], c.v[3]);
    cswap_desc(c.v[0], c.v[1]);
    cswap_desc(c.v[2], c.v[3]);
    return c;
}
__device__ __forceinline__ void top4_insert(Top4& t, float x) {
    if (!(x > t.v[3])) return;
    t.v[3] = x;
    cswap_desc(t.v[2], t.v[3]);
    cswap_desc(t.v[1], t.v[2]);
    cswap_desc(t.v[0], t.v[1]);
}
__device__ __forceinline__ Top4 top4_shfl_up(const Top4& t, int d) {
    Top4 r;
#pragma unroll
    for (int i = 0; i < 4; ++i) r.v[i] = __shfl_up_sync(0xffffffffu, t.v[i], d);
    return r;
}

struct ProbeCtx {
    const DCollider* ca;
    const DCollider* cb;
    F3 pa, pb;
    Qt qa, qb, qna, qnb;
    float vs_a, vs_b, spec;
};

// The 27 neighbour offsets in checkNeighborhood order: dz, dy, dx in {-1,0,1}.
__device__ __forceinline__ I3 probe_offset(uint32_t k) {
    return I3{(int32_t)(k % 3u) - 1, (int32_t)((k / 3u) % 3u) - 1, (int32_t)(k / 9u) - 1};
}

// Penetration of a distance-passing candidate (generateContact).
__device__ __forceinline__ float cand_pen(float vs_a, uint32_t ta, uint32_t tb, float d2) {
    float pen = vs_a - sqrtf(d2);
    if (ta == kInside || tb == kInside) pen = fmaxf(pen, vs_a);
    return pen;
}

// generateContact (narrow_phase.zig:860-922).
__device__ void generate_contact(const ProbeCtx& c, uint32_t va, I3 ia, F3 wa, uint32_t vb, I3 ib, F3 wb,
                                 ContactRec* out) {
    const F3 diff = wb - wa;
    const float d2 = lensq3(diff);
    const float dist = sqrtf(d2);
    const F3 cp = (wa + wb) * 0.5f;
    float pen = c.vs_a - dist;
    const F3 na = qrotate(c.qa, lut_normal(vnormal(va)));
    const F3 nb = qrotate(c.qb, lut_normal(vnormal(vb)));
    F3 n;
    if (vtype(va) == kFace) {
        n = na;
    } else if (vtype(vb) == kFace) {
        n = -nb;
    } else if (dist > 0.001f) {
        const F3 dn = diff * (1.0f / dist);
        if (dot3(dn, na) > 0.3f) n = na;
        else if (dot3(dn, -nb) > 0.3f) n = -nb;
        else n = dn;
    } else {
        n = na;
    }
    if (vtype(va) == kInside || vtype(vb) == kInside) pen = fmaxf(pen, c.vs_a);
    const F3 la = inverse_transform_point(c.pa, c.qa, cp);
    const F3 lb = inverse_transform_point(c.pb, c.qb, cp);
    out->point[0] = cp.x; out->point[1] = cp.y; out->point[2] = cp.z;
    out->normal[0] = n.x; out->normal[1] = n.y; out->normal[2] = n.z;
    out->penetration = pen;
    out->la[0] = la.x; out->la[1] = la.y; out->la[2] = la.z;
    out->lb[0] = lb.x; out->lb[1] = lb.y; out->lb[2] = lb.z;
    out->normal_impulse = 0.f;
    out->tangent_impulse[0] = 0.f;
    out->tangent_impulse[1] = 0.f;
    out->normal_mass = 0.f;
    out->tangent_mass[0] = 0.f;
    out->tangent_mass[1] = 0.f;
    out->_pad = 0u;
    out->feature_id = feature_id(ia, ib);
}

// checkNeighborhood (narrow_phase.zig:796-857) for one A voxel: its 27
// probes in dz, dy, dx order, clipped to B's voxel bounds first (a probe
// outside them is skipped, isValidCoord); for each non-empty B voxel the
// type filter, the distance test and, for a pass, the candidate's penetration
// into the lane's top-4 and its bit (dz*9 + dy*3 + dx, offsets from -1) into
// the mask.
__device__ __forceinline__ int32_t clip_lo(int32_t bound, int32_t centre) {
    const long long d = (long long)bound - (long long)centre;
    return d > -1 ? (d > 2 ? 2 : (int32_t)d) : -1;
}
__device__ __forceinline__ int32_t clip_hi(int32_t bound_excl, int32_t centre) {
    const long long d = (long long)bound_excl - 1ll - (long long)centre;
    return d < 1 ? (d < -2 ? -2 : (int32_t)d) : 1;
}
__device__ __forceinline__ void probe_neighbourhood(WorldDev& w, const ColliderSet& cs, const ProbeCtx& c, uint32_t p,
                                                    uint32_t ta, int32_t x, int32_t y, int32_t z, F3 wa, I3 cbv,
                                                    uint32_t* mask, Top4* t, uint32_t* checked) {
    const DCollider& cb = *c.cb;
    if (cb.nb_off != kNoTable) {
        // one lookup gives the non-empty probes (counted as checked) and those
        // passing type_filter(ta, tb) (ta is never empty here); only the
        // latter are transformed and distance-tested, in probe order.  A
        // centre outside [min_bound - 1, max_bound] has no neighbour in bounds.
        const uint32_t ex = (uint32_t)(cb.max_bound[0] - cb.min_bound[0]) + 2u,
                       ey = (uint32_t)(cb.max_bound[1] - cb.min_bound[1]) + 2u,
                       ez = (uint32_t)(cb.max_bound[2] - cb.min_bound[2]) + 2u;
        const uint32_t tx = (uint32_t)cbv.x - ((uint32_t)cb.min_bound[0] - 1u),
                       ty = (uint32_t)cbv.y - ((uint32_t)cb.min_bound[1] - 1u),
                       tz = (uint32_t)cbv.z - ((uint32_t)cb.min_bound[2] - 1u);
        if (tx >= ex || ty >= ey || tz >= ez) return;
        const uint4 nm = __ldg(cs.nb + cb.nb_off + (tx + ex * (ty + ey * tz)));
        *checked += (uint32_t)__popc(nm.x);
        const uint32_t ps = ta == kCorner ? nm.x : (ta == kEdge ? nm.z : nm.y);
        for (uint32_t m = ps; m; m &= m - 1u) {
            const uint32_t k = __ffs(m) - 1;
            const I3 o = probe_offset(k);
            const int32_t bx = cbv.x + o.x, by = cbv.y + o.y, bz = cbv.z + o.z;
            const F3 wb = transform_point_n(c.pb, c.qnb, voxel_to_local(c.vs_b, bx, by, bz));
            const F3 diff = wb - wa;
            const float d2 = lensq3(diff);
            const bool pass = d2 < c.spec;
            if (w.cfg.dump_candidates) {
                const uint32_t slot = atomicAdd(&w.ctr[C_DUMP_N], 1u);
                if (slot < w.dump_cap) {
                    WorldDev::Cand& r = w.dump[slot];
                    r.pair_index = p;
                    r.a[0] = x; r.a[1] = y; r.a[2] = z;
                    r.b[0] = bx; r.b[1] = by; r.b[2] = bz;
                    r.passed = pass ? 1u : 0u;
                    r.dist_sq = d2;
                }
            }
            if (pass) {
                *mask |= 1u << k;
                top4_insert(*t, cand_pen(c.vs_a, ta, ((nm.w >> k) & 1u) ? (uint32_t)kInside : (uint32_t)kCorner, d2));
            }
        }
        return;
    }
    const int32_t lx = clip_lo(cb.min_bound[0], cbv.x), hx = clip_hi(cb.max_bound[0], cbv.x);
    const int32_t ly = clip_lo(cb.min_bound[1], cbv.y), hy = clip_hi(cb.max_bound[1], cbv.y);
    const int32_t lz = clip_lo(cb.min_bound[2], cbv.z), hz = clip_hi(cb.max_bound[2], cbv.z);
    if (lx > hx || ly > hy || lz > hz) return;
    // the brick holding the centre voxel (every probe is inside B's voxel
    // bounds, so inside its brick grid): probes in the same brick read their
    // byte at a fixed offset from the centre's, the others look their brick up
    const int32_t cx = cbv.x & 7, cy = cbv.y & 7, cz = cbv.z & 7;
    const int32_t cslot = brick_slot(cs, cb, cbv.x >> 3, cbv.y >> 3, cbv.z >> 3);
    const uint8_t* cvox = cs.vox + (size_t)(cb.brick_off + (uint32_t)max(cslot, 0)) * 512u +
                          (uint32_t)(cx + 8 * cy + 64 * cz);
    for (int32_t dz = lz; dz <= hz; ++dz)
        for (int32_t dy = ly; dy <= hy; ++dy)
            for (int32_t dx = lx; dx <= hx; ++dx) {
                const uint32_t k = (uint32_t)((dz + 1) * 9 + (dy + 1) * 3 + (dx + 1));
                const int32_t bx = cbv.x + dx, by = cbv.y + dy, bz = cbv.z + dz;
                const bool same = (uint32_t)(cx + dx) < 8u && (uint32_t)(cy + dy) < 8u && (uint32_t)(cz + dz) < 8u;
                const uint32_t vb = same ? (cslot >= 0 ? (uint32_t)__ldg(cvox + (dx + 8 * dy + 64 * dz)) : 0u)
                                         : voxel_at(cs, cb, bx, by, bz);
                const uint32_t tb = vtype(vb);
                if (tb == kEmpty) continue;
                ++*checked;
                if (!type_filter(ta, tb)) continue;
                const F3 wb = transform_point_n(c.pb, c.qnb, voxel_to_local(c.vs_b, bx, by, bz));
                const F3 diff = wb - wa;
                const float d2 = lensq3(diff);
                const bool pass = d2 < c.spec;
                if (w.cfg.dump_candidates) {
                    const uint32_t slot = atomicAdd(&w.ctr[C_DUMP_N], 1u);
                    if (slot < w.dump_cap) {
                        WorldDev::Cand& r = w.dump[slot];
                        r.pair_index = p;
                        r.a[0] = x; r.a[1] = y; r.a[2] = z;
                        r.b[0] = bx; r.b[1] = by; r.b[2] = bz;
                        r.passed = pass ? 1u : 0u;
                        r.dist_sq = d2;
                    }
                }
                if (pass) {
                    *mask |= 1u << k;
                    top4_insert(*t, cand_pen(c.vs_a, ta, tb, d2));
                }
            }
}

// A candidate entering the manifold during detection: penetration, feature
// id, and where it came from (A voxel li of the region in loop order, probe
// k).  Its contact is built only if it is still in the manifold when the pair
// ends: a contact's fields are a function of (li, k), and the impulses of
// every contact added during detection are zero.
struct CandRec {
    unsigned long long fid;
    float pen;
    uint32_t li, k, _pad;
};

// Entering candidates a warp lists at once before lane 0 applies them.
constexpr uint32_t kWarpReplay = 16;

// Per-warp shared state of phase_probe.
struct WarpManifold {
    ContactRec c[4];              // the pair's contacts, built when it ends
    CandRec k[4];                 // the manifold during detection
    CandRec list[kWarpReplay];
    float pens[4];
    uint32_t n;
    uint32_t pad[3];
};

// ContactManifold.addContact (narrow_phase.zig:451-481) on candidate
// records, executed by one lane: a contact with the same feature id is
// replaced (keeping its impulses, all zero here), else appended while fewer
// than four, else the first contact of least penetration below the new one
// is replaced.
__device__ __forceinline__ void add_cand(WarpManifold& m, const CandRec& r) {
    for (uint32_t i = 0; i < m.n; ++i) {
        if (m.k[i].fid == r.fid) {
            m.k[i] = r;
            return;
        }
    }
    if (m.n < 4u) {
        m.k[m.n] = r;
        m.n += 1u;
        return;
    }
    float mp = r.pen;
    int mi = -1;
    for (uint32_t i = 0; i < m.n; ++i) {
        if (m.k[i].pen < mp) {
            mp = m.k[i].pen;
            mi = (int)i;
        }
    }
    if (mi >= 0) m.k[mi] = r;
}
// The manifold's penetration multiset (at most four finite values, so every
// insert lands), by one lane, into m.pens.
__device__ __forceinline__ void cand_pens(WarpManifold& m) {
    Top4 s = top4_empty();
    for (uint32_t i = 0; i < m.n; ++i) top4_insert(s, m.k[i].pen);
    m.pens[0] = s.v[0];
    m.pens[1] = s.v[1];
    m.pens[2] = s.v[2];
    m.pens[3] = s.v[3];
}
// generateContact for candidate r of the pair probed with c over the region
// starting at rmin, nx x ny voxels per z layer: the same lookups and
// transforms as the detection loop.
__device__ void build_contact(const ColliderSet& cs, const ProbeCtx& c, const int32_t* rmin, uint32_t nx,
                              uint32_t ny, const CandRec& r, ContactRec* out) {
    const int32_t x = rmin[0] + (int32_t)(r.li % nx), y = rmin[1] + (int32_t)((r.li / nx) % ny),
                  z = rmin[2] + (int32_t)(r.li / (nx * ny));
    const uint32_t va = voxel_at(cs, *c.ca, x, y, z);
    const F3 wa = transform_point_n(c.pa, c.qna, voxel_to_local(c.vs_a, x, y, z));
    const I3 cbv = local_to_voxel(c.vs_b, inverse_transform_point(c.pb, c.qb, wa));
    const I3 o = probe_offset(r.k);
    const I3 ibv{cbv.x + o.x, cbv.y + o.y, cbv.z + o.z};
    const uint32_t vb = voxel_at(cs, *c.cb, ibv.x, ibv.y, ibv.z);
    const F3 wb = transform_point_n(c.pb, c.qnb, voxel_to_local(c.vs_b, ibv.x, ibv.y, ibv.z));
    generate_contact(c, va, I3{x, y, z}, wa, vb, ibv, wb, out);
}

// One warp runs detectVoxelCollisions for pair p.  The inclusive z, y, x loop
// over the overlap region is cut into groups of 32 consecutive voxels, one per
// lane; each lane runs the 27 probes of its voxel.  The manifold reduction is
// order dependent, so it is reproduced exactly: a candidate can only enter the
// 4-slot manifold if its penetration beats the 4th largest penetration of all
// candidates before it (the multiset of penetrations held by the manifold is
// always the top four of the prefix).  A warp scan of top-4 multisets gives
// every lane that prefix, seeded with the manifold's state; only the entering
// candidates are replayed, in order, through addContact.
__device__ void probe_pair(WorldDev& w, const ColliderSet& cs, uint32_t cur, uint32_t p, WarpManifold& sm) {
    const uint32_t lane = threadIdx.x & 31;
    PairInfo& pi = w.pinfo[p];
    const uint32_t ia = pi.ia, ib = pi.ib;
    const DBody& A = w.body[ia];
    const DBody& B = w.body[ib];
    const DBodyProp& prA = w.prop[ia];
    const DBodyProp& prB = w.prop[ib];
    ProbeCtx c;
    c.ca = &cs.c[prA.collider];
    c.cb = &cs.c[prB.collider];
    c.pa = f3of(A.p);
    c.pb = f3of(B.p);
    c.qa = qof(A.q);
    c.qb = qof(B.q);
    c.qna = qof(w.qn[ia]);
    c.qnb = qof(w.qn[ib]);
    c.vs_a = c.ca->vs;
    c.vs_b = c.cb->vs;
    {
        const float cds = c.vs_a * c.vs_a * 1.0f * 1.0f;
        c.spec = cds + 0.02f * 0.02f + 2.0f * sqrtf(cds) * 0.02f;
    }
    const DCollider& ca = *c.ca;
    const DCollider& cb = *c.cb;
    const int32_t nx = pi.rmax[0] - pi.rmin[0] + 1, ny = pi.rmax[1] - pi.rmin[1] + 1,
                  nz = pi.rmax[2] - pi.rmin[2] + 1;
    const unsigned long long V = (unsigned long long)nx * (unsigned long long)ny * (unsigned long long)nz;
    if (lane == 0) sm.n = 0u;
    Top4 state = top4_empty();
    uint32_t checked = 0, ncand = 0;
    if (w.cfg.count_bricks) {
        // traffic accounting: A bricks in the region, B bricks in B's region
        uint32_t nb = warp_count_bricks(cs, ca, I3{pi.rmin[0], pi.rmin[1], pi.rmin[2]},
                                        I3{pi.rmax[0], pi.rmax[1], pi.rmax[2]});
        I3 blo, bhi;
        if (overlap_region(cb, c.pb, c.qb, ca, c.pa, c.qa, &blo, &bhi)) nb += warp_count_bricks(cs, cb, blo, bhi);
        if (lane == 0) atomicAdd(&w.ctr[C_BRICKS], nb);
    }
    __syncwarp();
    for (unsigned long long base = 0; base < V; base += 32ull) {
        const unsigned long long l = base + lane;
        uint32_t va = 0u;
        int32_t x = 0, y = 0, z = 0;
        if (l < V) {
            const uint32_t li = (uint32_t)l;
            x = pi.rmin[0] + (int32_t)(li % (uint32_t)nx);
            y = pi.rmin[1] + (int32_t)((li / (uint32_t)nx) % (uint32_t)ny);
            z = pi.rmin[2] + (int32_t)(li / ((uint32_t)nx * (uint32_t)ny));
            va = voxel_at(cs, ca, x, y, z);
        }
        uint32_t mask = 0u;
        Top4 t = top4_empty();
        F3 wa{0.f, 0.f, 0.f};
        I3 cbv{0, 0, 0};
        const uint32_t ta = vtype(va);
        if (ta != kEmpty) {
            wa = transform_point_n(c.pa, c.qna, voxel_to_local(c.vs_a, x, y, z));
            cbv = local_to_voxel(c.vs_b, inverse_transform_point(c.pb, c.qb, wa));
            probe_neighbourhood(w, cs, c, p, ta, x, y, z, wa, cbv, &mask, &t, &checked);
        }
        if (__ballot_sync(0xffffffffu, mask != 0u) == 0u) continue;
        ncand += __popc(mask);
        // a candidate enters only above the running 4th penetration, which is
        // at least the manifold's: when no lane's best beats that, none does
        if (__ballot_sync(0xffffffffu, t.v[0] > state.v[3]) == 0u) continue;
        // exclusive warp scan of the lanes' top-4 multisets
        Top4 inc = t;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const Top4 o = top4_shfl_up(inc, d);
            if ((int)lane >= d) inc = top4_merge(o, inc);
        }
        Top4 ex = top4_shfl_up(inc, 1);
        if (lane == 0) ex = top4_empty();
        Top4 run = top4_merge(state, ex);
        // candidates of this lane that enter the manifold
        uint32_t enter = 0u;
        for (uint32_t mm = mask; mm; mm &= mm - 1u) {
            const uint32_t k = __ffs(mm) - 1;
            const I3 o = probe_offset(k);
            const int32_t bx = cbv.x + o.x, by = cbv.y + o.y, bz = cbv.z + o.z;
            const uint32_t vb = voxel_at(cs, cb, bx, by, bz);
            const F3 wb = transform_point_n(c.pb, c.qnb, voxel_to_local(c.vs_b, bx, by, bz));
            const float d2 = lensq3(wb - wa);
            const float pen = cand_pen(c.vs_a, ta, vtype(vb), d2);
            if (pen > run.v[3]) {
                enter |= 1u << k;
                top4_insert(run, pen);
            }
        }
        // entering candidates in canonical order (lane = voxel order, then
        // probe order): the lanes list them at once, kWarpReplay at a time;
        // lane 0 applies them in list order
        const uint32_t ne = (uint32_t)__popc(enter);
        const uint32_t ninc = warp_incl_scan(ne);
        const uint32_t total = __shfl_sync(0xffffffffu, ninc, 31);
        for (uint32_t lo = 0; lo < total; lo += kWarpReplay) {
            uint32_t e = ninc - ne;
            for (uint32_t mm = enter; mm; mm &= mm - 1u, ++e) {
                if (e < lo || e >= lo + kWarpReplay) continue;
                const uint32_t k = __ffs(mm) - 1;
                const I3 o = probe_offset(k);
                const I3 ibv{cbv.x + o.x, cbv.y + o.y, cbv.z + o.z};
                const uint32_t vb = voxel_at(cs, cb, ibv.x, ibv.y, ibv.z);
                const F3 wb = transform_point_n(c.pb, c.qnb, voxel_to_local(c.vs_b, ibv.x, ibv.y, ibv.z));
                CandRec& r = sm.list[e - lo];
                r.fid = feature_id(I3{x, y, z}, ibv);
                r.pen = cand_pen(c.vs_a, ta, vtype(vb), lensq3(wb - wa));
                r.li = (uint32_t)l;
                r.k = k;
                r._pad = 0u;
            }
            __syncwarp();
            if (lane == 0) {
                const uint32_t cnt = min(kWarpReplay, total - lo);
                for (uint32_t i = 0; i < cnt; ++i) add_cand(sm, sm.list[i]);
            }
            __syncwarp();
        }
        // manifold penetration multiset -> state
        if (lane == 0) cand_pens(sm);
        __syncwarp();
        state.v[0] = sm.pens[0];
        state.v[1] = sm.pens[1];
        state.v[2] = sm.pens[2];
        state.v[3] = sm.pens[3];
    }
    checked = warp_sum(checked);
    ncand = warp_sum(ncand);
    // the contacts left in the manifold
    if (lane < sm.n) build_contact(cs, c, pi.rmin, (uint32_t)nx, (uint32_t)ny, sm.k[lane], &sm.c[lane]);
    __syncwarp();
    ManifoldRec& out = w.man[cur][p];
    if (lane == 0) {
        pi.voxels_checked = checked;
        pi.candidates = ncand;
        out.a = prA.id;
        out.b = prB.id;
        out.n = sm.n;
        out.friction = sqrtf(prA.friction * prB.friction);
        out.restitution = fmaxf(prA.restitution, prB.restitution);
        out._pad = 0u;
    }
    __syncwarp();
    // copy the contacts (one lane per 4-byte word)
    const uint32_t words = sm.n * (uint32_t)(sizeof(ContactRec) / 4);
    const uint32_t* src = reinterpret_cast<const uint32_t*>(sm.c);
    uint32_t* dst = reinterpret_cast<uint32_t*>(out.c);
    for (uint32_t i = lane; i < words; i += 32u) dst[i] = src[i];
    __syncwarp();
}

// The same narrow phase for one pair with a large overlap region, run by the
// whole CTA: each pass covers blockDim.x consecutive voxels of the inclusive
// z, y, x loop (one per thread).  The manifold's order-dependent reduction is
// reproduced as in probe_pair, with a CTA-wide exclusive scan of the
// threads' top-4 multisets in voxel order; the threads build the contacts
// that enter, and one thread adds them to the manifold in that order.
constexpr uint32_t kBlockReplay = 64;
__device__ void probe_pair_block(WorldDev& w, const ColliderSet& cs, uint32_t cur, uint32_t p, WarpManifold& sm) {
    __shared__ Top4 s_top[32];
    __shared__ CandRec s_rec[kBlockReplay];
    const uint32_t tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nwarps = blockDim.x >> 5;
    PairInfo& pi = w.pinfo[p];
    const uint32_t ia = pi.ia, ib = pi.ib;
    const DBody& A = w.body[ia];
    const DBody& B = w.body[ib];
    const DBodyProp& prA = w.prop[ia];
    const DBodyProp& prB = w.prop[ib];
    ProbeCtx c;
    c.ca = &cs.c[prA.collider];
    c.cb = &cs.c[prB.collider];
    c.pa = f3of(A.p);
    c.pb = f3of(B.p);
    c.qa = qof(A.q);
    c.qb = qof(B.q);
    c.qna = qof(w.qn[ia]);
    c.qnb = qof(w.qn[ib]);
    c.vs_a = c.ca->vs;
    c.vs_b = c.cb->vs;
    {
        const float cds = c.vs_a * c.vs_a * 1.0f * 1.0f;
        c.spec = cds + 0.02f * 0.02f + 2.0f * sqrtf(cds) * 0.02f;
    }
    const DCollider& ca = *c.ca;
    const DCollider& cb = *c.cb;
    const int32_t nx = pi.rmax[0] - pi.rmin[0] + 1, ny = pi.rmax[1] - pi.rmin[1] + 1,
                  nz = pi.rmax[2] - pi.rmin[2] + 1;
    const unsigned long long V = (unsigned long long)nx * (unsigned long long)ny * (unsigned long long)nz;
    if (tid == 0) sm.n = 0u;
    if (wid == 0 && w.cfg.count_bricks) {
        // traffic accounting: A bricks in the region, B bricks in B's region
        uint32_t nb = warp_count_bricks(cs, ca, I3{pi.rmin[0], pi.rmin[1], pi.rmin[2]},
                                        I3{pi.rmax[0], pi.rmax[1], pi.rmax[2]});
        I3 blo, bhi;
        if (overlap_region(cb, c.pb, c.qb, ca, c.pa, c.qa, &blo, &bhi)) nb += warp_count_bricks(cs, cb, blo, bhi);
        if (lane == 0) atomicAdd(&w.ctr[C_BRICKS], nb);
    }
    __syncthreads();
    Top4 state = top4_empty();
    uint32_t checked = 0, ncand = 0;
    for (unsigned long long base = 0; base < V; base += blockDim.x) {
        const unsigned long long l = base + tid;
        uint32_t va = 0u;
        int32_t x = 0, y = 0, z = 0;
        if (l < V) {
            const uint32_t li = (uint32_t)l;
            x = pi.rmin[0] + (int32_t)(li % (uint32_t)nx);
            y = pi.rmin[1] + (int32_t)((li / (uint32_t)nx) % (uint32_t)ny);
            z = pi.rmin[2] + (int32_t)(li / ((uint32_t)nx * (uint32_t)ny));
            va = voxel_at(cs, ca, x, y, z);
        }
        uint32_t mask = 0u;
        Top4 t = top4_empty();
        F3 wa{0.f, 0.f, 0.f};
        I3 cbv{0, 0, 0};
        const uint32_t ta = vtype(va);
        if (ta != kEmpty) {
            wa = transform_point_n(c.pa, c.qna, voxel_to_local(c.vs_a, x, y, z));
            cbv = local_to_voxel(c.vs_b, inverse_transform_point(c.pb, c.qb, wa));
            probe_neighbourhood(w, cs, c, p, ta, x, y, z, wa, cbv, &mask, &t, &checked);
        }
        if (!__syncthreads_or(mask != 0u)) continue;
        ncand += __popc(mask);
        // a candidate enters only above the running 4th penetration, which is
        // at least the manifold's: when no thread's best beats that, none does
        if (!__syncthreads_or(t.v[0] > state.v[3])) continue;
        // CTA-wide exclusive scan of the threads' top-4 multisets
        Top4 inc = t;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const Top4 o = top4_shfl_up(inc, d);
            if ((int)lane >= d) inc = top4_merge(o, inc);
        }
        if (lane == 31) s_top[wid] = inc;
        __syncthreads();
        if (wid == 0) {
            Top4 wi = lane < nwarps ? s_top[lane] : top4_empty();
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const Top4 o = top4_shfl_up(wi, d);
                if ((int)lane >= d) wi = top4_merge(o, wi);
            }
            Top4 we = top4_shfl_up(wi, 1);
            if (lane == 0) we = top4_empty();
            if (lane < nwarps) s_top[lane] = we;
        }
        __syncthreads();
        Top4 ex = top4_shfl_up(inc, 1);
        if (lane == 0) ex = top4_empty();
        Top4 run = top4_merge(state, top4_merge(s_top[wid], ex));
        // candidates of this thread that enter the manifold
        uint32_t enter = 0u;
        for (uint32_t mm = mask; mm; mm &= mm - 1u) {
            const uint32_t k = __ffs(mm) - 1;
            const I3 o = probe_offset(k);
            const int32_t bx = cbv.x + o.x, by = cbv.y + o.y, bz = cbv.z + o.z;
            const uint32_t vb = voxel_at(cs, cb, bx, by, bz);
            const F3 wb = transform_point_n(c.pb, c.qnb, voxel_to_local(c.vs_b, bx, by, bz));
            const float d2 = lensq3(wb - wa);
            const float pen = cand_pen(c.vs_a, ta, vtype(vb), d2);
            if (pen > run.v[3]) {
                enter |= 1u << k;
                top4_insert(run, pen);
            }
        }
        // entering candidates in (voxel, probe) order: the threads list them
        // at once, kBlockReplay at a time, into s_rec; thread 0 applies them
        // in that order
        uint32_t total = 0;
        const uint32_t off = block_excl_scan((uint32_t)__popc(enter), &total);
        for (uint32_t lo = 0; lo < total; lo += kBlockReplay) {
            uint32_t e = off;
            for (uint32_t mm = enter; mm; mm &= mm - 1u, ++e) {
                if (e < lo || e >= lo + kBlockReplay) continue;
                const uint32_t k = __ffs(mm) - 1;
                const I3 o = probe_offset(k);
                const I3 ibv{cbv.x + o.x, cbv.y + o.y, cbv.z + o.z};
                const uint32_t vb = voxel_at(cs, cb, ibv.x, ibv.y, ibv.z);
                const F3 wb = transform_point_n(c.pb, c.qnb, voxel_to_local(c.vs_b, ibv.x, ibv.y, ibv.z));
                CandRec& r = s_rec[e - lo];
                r.fid = feature_id(I3{x, y, z}, ibv);
                r.pen = cand_pen(c.vs_a, ta, vtype(vb), lensq3(wb - wa));
                r.li = (uint32_t)l;
                r.k = k;
                r._pad = 0u;
            }
            __syncthreads();
            if (tid == 0) {
                const uint32_t cnt = min(kBlockReplay, total - lo);
                for (uint32_t i = 0; i < cnt; ++i) add_cand(sm, s_rec[i]);
            }
            __syncthreads();
        }
        // manifold penetration multiset -> state
        if (tid == 0) cand_pens(sm);
        __syncthreads();
        state.v[0] = sm.pens[0];
        state.v[1] = sm.pens[1];
        state.v[2] = sm.pens[2];
        state.v[3] = sm.pens[3];
    }
    checked = block_sum(checked);
    ncand = block_sum(ncand);
    // the contacts left in the manifold
    if (tid < sm.n) build_contact(cs, c, pi.rmin, (uint32_t)nx, (uint32_t)ny, sm.k[tid], &sm.c[tid]);
    __syncthreads();
    ManifoldRec& out = w.man[cur][p];
    if (tid == 0) {
        pi.voxels_checked = checked;
        pi.candidates = ncand;
        out.a = prA.id;
        out.b = prB.id;
        out.n = sm.n;
        out.friction = sqrtf(prA.friction * prB.friction);
        out.restitution = fmaxf(prA.restitution, prB.restitution);
        out._pad = 0u;
    }
    __syncthreads();
    const uint32_t words = sm.n * (uint32_t)(sizeof(ContactRec) / 4);
    const uint32_t* src = reinterpret_cast<const uint32_t*>(sm.c);
    uint32_t* dst = reinterpret_cast<uint32_t*>(out.c);
    for (uint32_t i = tid; i < words; i += blockDim.x) dst[i] = src[i];
    __syncthreads();
}

template <class G>
__device__ bool phase_probe(G& g, WorldDev& w, const ColliderSet& cs, uint32_t cur, WarpManifold* warp_sm,
                            const CacheSmem& csm) {
    const uint32_t lane = threadIdx.x & 31;
    WarpManifold& sm = warp_sm[threadIdx.x >> 5];
    // the cache lookups are replayed by one CTA of a grid (which detects
    // nothing: the replay is a chain of dependent rounds, and other work on
    // its SM would slow it more than it is worth), or by one warp of a lone
    // CTA while its other warps start detecting at once
    const bool replay_cta = w.cfg.use_cache && g.nblocks() > 1u && g.block() == 0u;
    if (replay_cta && w.cache_cap >= 64u * 16u &&
        (size_t)(blockDim.x >> 5) * sizeof(WarpManifold) >= cta_replay_scratch_bytes()) {
        cache_replay_cta(w, csm, reinterpret_cast<unsigned char*>(warp_sm));
        return g.sync();
    }
    if (w.cfg.use_cache && g.rank() < 32u) cache_replay(w, csm);
    // large regions first, one CTA each, then the rest one warp each
    const uint32_t nh = *(volatile uint32_t*)&w.ctr[C_NHEAVY];
    if (replay_cta) return g.sync();
    if (nh) {
        __shared__ uint32_t s_h;
        for (;;) {
            __syncthreads();
            if (threadIdx.x == 0) s_h = atomicAdd(&w.ctr[C_HWORK], 1u);
            __syncthreads();
            const uint32_t h = s_h;
            if (h >= nh) break;
            probe_pair_block(w, cs, cur, w.cons[h], warp_sm[0]);
        }
    }
    for (;;) {
        uint32_t p = 0;
        if (lane == 0) p = atomicAdd(&w.ctr[C_WORK], 1u);
        p = __shfl_sync(0xffffffffu, p, 0);
        if (p >= w.n_pairs) break;
        const uint32_t fl = w.pinfo[p].flags;
        if ((fl & (PF_DETECT | PF_CACHE)) && (fl & PF_REGION) && !(fl & PF_HEAVY)) probe_pair(w, cs, cur, p, sm);
    }
    return g.sync();
}

// ---------------------------------------------------------------------------
// Phase: finalize (cache hits, carries, ContactManager.addManifold warm start)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void warm_from_prev(const WorldDev& w, uint32_t prev, ManifoldRec& m) {
    const uint32_t idx = ht_find(w.ht[prev], w.ht_cap, pair_key(m.a, m.b));
    if (idx == 0xFFFFFFFFu) return;
    const ManifoldRec& o = w.man[prev][idx];
    for (uint32_t i = 0; i < m.n; ++i)
        for (uint32_t j = 0; j < o.n; ++j)
            if (m.c[i].feature_id == o.c[j].feature_id) {
                m.c[i].normal_impulse = o.c[j].normal_impulse;
                m.c[i].tangent_impulse[0] = o.c[j].tangent_impulse[0];
                m.c[i].tangent_impulse[1] = o.c[j].tangent_impulse[1];
                break;
            }
}

template <class G>
__device__ bool phase_finalize(G& g, WorldDev& w, uint32_t cur, uint32_t prev) {
    uint32_t skipped = 0, colliding = 0, contacts = 0, voxels = 0, manifolds = 0, cands = 0;
    for (uint32_t p = g.rank(); p < w.n_pairs; p += g.size()) {
        const PairInfo& pi = w.pinfo[p];
        const uint32_t fl = pi.flags;
        ManifoldRec& m = w.man[cur][p];
        if (fl & PF_CARRY) {
            ++skipped;
            const uint2 pr = w.pairs[p];
            const uint32_t idx = ht_find(w.ht[prev], w.ht_cap, pair_key(pr.x, pr.y));
            if (idx != 0xFFFFFFFFu) m = w.man[prev][idx];
            else m.n = 0u;
        } else if (!(fl & PF_TESTED) || (fl & (PF_NOCOLL | PF_SEPARATED))) {
            m.n = 0u;
        } else if ((fl & PF_CACHE) && pi.hit == 1u) {
            const CacheValRec& v = w.cval[pi.cache_slot];
            if (v.has_collision) {
                const DBodyProp& a = w.prop[pi.ia];
                const DBodyProp& b = w.prop[pi.ib];
                m.a = a.id;
                m.b = b.id;
                m.friction = sqrtf(a.friction * b.friction);
                m.restitution = fmaxf(a.restitution, b.restitution);
                m._pad = 0u;
                // ContactManifold.addContact from empty: feature ids are unique
                m.n = 0u;
                for (uint32_t i = 0; i < v.n; ++i) {
                    bool dup = false;
                    for (uint32_t j = 0; j < m.n; ++j)
                        if (m.c[j].feature_id == v.c[i].feature_id) {
                            const float ni = m.c[j].normal_impulse, t0 = m.c[j].tangent_impulse[0],
                                        t1 = m.c[j].tangent_impulse[1];
                            m.c[j] = v.c[i];
                            m.c[j].normal_impulse = ni;
                            m.c[j].tangent_impulse[0] = t0;
                            m.c[j].tangent_impulse[1] = t1;
                            dup = true;
                            break;
                        }
                    if (!dup && m.n < 4u) m.c[m.n++] = v.c[i];
                }
                ++colliding;
                contacts += v.n;
                voxels += v.voxels_checked;
                warm_from_prev(w, prev, m);
            } else {
                m.n = 0u;
            }
        } else if ((fl & PF_DETECT) || (fl & PF_CACHE)) {
            if (!(fl & PF_REGION)) {
                const DBodyProp& a = w.prop[pi.ia];
                const DBodyProp& b = w.prop[pi.ib];
                m.a = a.id;
                m.b = b.id;
                m.n = 0u;
                m.friction = sqrtf(a.friction * b.friction);
                m.restitution = fmaxf(a.restitution, b.restitution);
            }
            voxels += pi.voxels_checked;
            cands += pi.candidates;
            if (m.n > 0u) {
                ++colliding;
                contacts += m.n;
                warm_from_prev(w, prev, m);
            }
        } else {
            m.n = 0u;
        }
        if (m.n > 0u) {
            ++manifolds;
            ht_insert(w.ht[cur], w.ht_cap, pair_key(m.a, m.b), p);
        }
    }
    skipped = warp_sum(skipped);
    colliding = warp_sum(colliding);
    contacts = warp_sum(contacts);
    voxels = warp_sum(voxels);
    manifolds = warp_sum(manifolds);
    cands = warp_sum(cands);
    if ((threadIdx.x & 31) == 0) {
        if (skipped) atomicAdd(&w.ctr[C_SKIPPED_SLEEPING], skipped);
        if (colliding) atomicAdd(&w.ctr[C_PAIRS_COLLIDING], colliding);
        if (contacts) atomicAdd(&w.ctr[C_CONTACTS], contacts);
        if (voxels) atomicAdd(&w.ctr[C_VOXELS_CHECKED], voxels);
        if (manifolds) atomicAdd(&w.ctr[C_MANIFOLDS], manifolds);
        if (cands) atomicAdd(&w.ctr[C_CANDIDATES], cands);
    }
    if (!g.sync()) return false;
    // BrickPairCache.put values of this frame's misses (last writer wins)
    if (w.cfg.use_cache) {
        for (uint32_t p = g.rank(); p < w.n_pairs; p += g.size()) {
            const PairInfo& pi = w.pinfo[p];
            if (!(pi.flags & PF_CACHE) || pi.hit != 2u) continue;
            if (pi.flags & (PF_NOCOLL | PF_SEPARATED)) continue;
            const uint32_t s = pi.cache_slot;
            if (s == 0xFFFFFFFFu || w.cwriter[s] != p) continue;
            const ManifoldRec& m = w.man[cur][p];
            CacheValRec& v = w.cval[s];
            const uint32_t n = m.n < 4u ? m.n : 4u;
            v.n = n;
            v.has_collision = n > 0u ? 1u : 0u;
            v.voxels_checked = pi.voxels_checked;
            for (uint32_t i = 0; i < n; ++i) {
                v.c[i] = m.c[i];
                v.c[i].normal_impulse = 0.f;
                v.c[i].tangent_impulse[0] = 0.f;
                v.c[i].tangent_impulse[1] = 0.f;
                v.c[i].normal_mass = 0.f;
                v.c[i].tangent_mass[0] = 0.f;
                v.c[i].tangent_mass[1] = 0.f;
            }
        }
    }
    return true;
}

// ---------------------------------------------------------------------------
// Phase: constraints (system.solve assembly, colouring, ContactSolver.addManifold)
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool writable(const DBodyProp& p) { return p.type == 2u && p.sleeping == 0u; }

// Jones-Plassmann priority; the oracle colours greedily in the same order.
__device__ __forceinline__ uint32_t jp_priority(uint32_t k) {
    uint32_t h = k * 0x9E3779B1u;
    h ^= h >> 16;
    h *= 0x85EBCA6Bu;
    h ^= h >> 13;
    h *= 0xC2B2AE35u;
    h ^= h >> 16;
    return h;
}
__device__ __forceinline__ bool jp_before(uint32_t i, uint32_t j) {
    const uint32_t pi = jp_priority(i), pj = jp_priority(j);
    return pi != pj ? pi > pj : i < j;
}
// Bound on the polling colouring's wait for higher-priority neighbours.
constexpr unsigned long long kColourTimeoutNs = 2000000000ull;

__device__ __forceinline__ size_t cpi(const WorldDev& w, uint32_t field, uint32_t slot, uint32_t pos) {
    return ((size_t)(field * 4u + slot)) * w.pair_cap + pos;
}

// ---------------------------------------------------------------------------
// Phase: islands (IslandManager.buildIslandsWithBodyTypes + updateSleepStates,
// islands.zig:318-495, run by system.solve before the solver, system.zig:705-760)
// ---------------------------------------------------------------------------
// The reference keeps only statistics from it (updateSleepStates reads copies
// of the bodies): islands, active and sleeping islands, the largest island.
// Islands are rebuilt when the frame's contact graph differs from the last
// build's.  The reference compares a 64-bit fold of the manifolds' pair keys
// in iteration order (computeGraphHash, islands.zig:277-296); here the key
// sequences themselves are compared, which differs only where two different
// sequences fold to the same hash.
// Build: union-find over the manifolds whose bodies are both non-static.  It
// is lock-free: a root is linked under the smaller root by CAS, so parents
// only point to smaller indices and an island's root is its smallest body
// index.  Every body a manifold names is in one island (a static body alone).
// Sleep: an island whose bodies are all still (|v|^2 and |w|^2 at most 0.1^2)
// for 0.5 s sleeps; for island body id k the k-th body of the table is read,
// as the reference indexes its body copies by id (islands.zig:437-440).

// The root of body i, halving the path on the way: each visited body is
// pointed at its grandparent, an ancestor in the same tree, so the trees stay
// valid while other threads link roots (a body that is no root never becomes
// one again, and only roots are linked).  Parents point to smaller indices,
// so the walk ends within i + 1 links.
__device__ __forceinline__ uint32_t isl_root(uint32_t* parent, uint32_t i) {
    uint32_t x = i;
    for (uint32_t k = 0; k <= i; ++k) {
        const uint32_t p = *(volatile uint32_t*)&parent[x];
        if (p == x) break;
        const uint32_t gp = *(volatile uint32_t*)&parent[p];
        if (gp != p) *(volatile uint32_t*)&parent[x] = gp;
        x = gp;
    }
    return x;
}
// UnionFind.unite: link the larger root under the smaller.  A failed CAS
// means another thread linked that root meanwhile; every link removes a
// root, so the retries are bounded by the body count.
__device__ __forceinline__ bool isl_unite(uint32_t* parent, uint32_t a, uint32_t b, uint32_t n) {
    for (uint32_t k = 0; k <= n; ++k) {
        a = isl_root(parent, a);
        b = isl_root(parent, b);
        if (a == b) return true;
        if (a < b) {
            const uint32_t t = a;
            a = b;
            b = t;
        }
        if (atomicCAS(&parent[a], a, b) == a) return true;
    }
    return false;
}

template <class G>
__device__ bool phase_islands(G& g, WorldDev& w, uint32_t cur, uint32_t* scratch) {
    if (!w.cfg.islands_on || !w.isl_state) return true;
    const uint32_t P = w.n_pairs, N = w.n_bodies;
    uint32_t* st = w.isl_state;
    const uint32_t buf = *(volatile uint32_t*)&st[IS_BUF] & 1u, nprev = *(volatile uint32_t*)&st[IS_NKEYS];
    const unsigned long long* kp = w.isl_keys[buf];
    unsigned long long* kc = w.isl_keys[buf ^ 1u];
    const ManifoldRec* man = w.man[cur];
    // 1. the frame's manifold keys in iteration order (pair order), against
    // the last build's
    uint32_t nm = 0;
    if (!group_scan(
            g, P, [&](uint32_t p) { return man[p].n > 0u ? 1u : 0u; },
            [&](uint32_t p, uint32_t q) {
                if (man[p].n == 0u) return;
                const unsigned long long k = pair_key(man[p].a, man[p].b);
                kc[q] = k;
                if (q >= nprev || kp[q] != k) atomicOr(&w.ctr[C_ISL_DIFF], 1u);
            },
            scratch, &nm))
        return false;
    const bool rebuild = *(volatile uint32_t*)&st[IS_DIRTY] != 0u || nm != nprev ||
                         *(volatile uint32_t*)&w.ctr[C_ISL_DIFF] != 0u || *(volatile uint32_t*)&st[IS_TOTAL] == 0u;
    if (!g.sync()) return false;  // every thread has decided before the state changes
    if (rebuild) {
        // 2. singletons, timers cleared (Island.clear)
        for (uint32_t i = g.rank(); i < N; i += g.size()) {
            w.isl_parent[i] = i;
            w.isl_flag[i] = 0u;
            w.isl_size[i] = 0u;
            w.isl_timer[i] = 0.0f;
        }
        if (g.rank() == 0) {
            st[IS_DIRTY] = 0u;
            st[IS_BUF] = buf ^ 1u;
            st[IS_NKEYS] = nm;
            st[IS_BUILDS] += 1u;
            st[IS_TOTAL] = 0u;
            st[IS_LARGEST] = 0u;
        }
        if (!g.sync()) return false;
        // 3. every body a manifold names; unions over non-static pairs
        bool ok = true;
        for (uint32_t p = g.rank(); p < P; p += g.size()) {
            if (man[p].n == 0u) continue;
            const uint32_t ia = w.pinfo[p].ia, ib = w.pinfo[p].ib;
            if (ia >= N || ib >= N) continue;
            atomicOr(&w.isl_flag[ia], ISL_TOUCHED);
            atomicOr(&w.isl_flag[ib], ISL_TOUCHED);
            if (w.prop[ia].type != 0u && w.prop[ib].type != 0u) ok &= isl_unite(w.isl_parent, ia, ib, N);
        }
        if (!ok) atomicOr(&w.ctr[C_ERROR], ERR_BOUNDS);
        if (!g.sync()) return false;
        // 4. each body's root, island sizes
        for (uint32_t i = g.rank(); i < N; i += g.size()) {
            if (!(w.isl_flag[i] & ISL_TOUCHED)) continue;
            const uint32_t r = isl_root(w.isl_parent, i);
            w.isl_parent[i] = r;
            atomicAdd(&w.isl_size[r], 1u);
        }
        if (!g.sync()) return false;
        // 5. the island count and the largest island
        uint32_t cnt = 0;
        for (uint32_t i = g.rank(); i < N; i += g.size()) {
            if ((w.isl_flag[i] & ISL_TOUCHED) && w.isl_parent[i] == i) {
                ++cnt;
                atomicMax(&st[IS_LARGEST], w.isl_size[i]);
            }
        }
        cnt = warp_sum(cnt);
        if ((threadIdx.x & 31u) == 0u && cnt) atomicAdd(&st[IS_TOTAL], cnt);
    } else if (g.rank() == 0) {
        st[IS_SKIPS] += 1u;
    }
    // 6. updateSleepStates: is every body of each island still?
    const float thr = 0.1f * 0.1f;  // ISLAND_SLEEP_{LINEAR,ANGULAR}_THRESHOLD squared
    for (uint32_t i = g.rank(); i < N; i += g.size()) {
        if (!(w.isl_flag[i] & ISL_TOUCHED)) continue;
        const uint32_t j = w.prop[i].id;
        if (j >= N || w.prop[j].type != 2u) continue;
        const DBody& b = w.body[j];
        if (lensq3(f3of(b.v)) > thr || lensq3(f3of(b.w)) > thr) atomicOr(&w.isl_flag[w.isl_parent[i]], ISL_MOVING);
    }
    if (!g.sync()) return false;
    // 7. per island: its timer and sleep flag
    uint32_t asleep = 0;
    for (uint32_t i = g.rank(); i < N; i += g.size()) {
        uint32_t f = w.isl_flag[i];
        if (!(f & ISL_TOUCHED) || w.isl_parent[i] != i) continue;
        if (!(f & ISL_MOVING)) {
            const float t = w.isl_timer[i] + w.cfg.dt;
            w.isl_timer[i] = t;
            if (t >= 0.5f) f |= ISL_ASLEEP;  // ISLAND_SLEEP_TIME_THRESHOLD
        } else {
            w.isl_timer[i] = 0.0f;
            f &= ~ISL_ASLEEP;
        }
        w.isl_flag[i] = f & ~ISL_MOVING;
        asleep += (f & ISL_ASLEEP) ? 1u : 0u;
    }
    asleep = warp_sum(asleep);
    if ((threadIdx.x & 31u) == 0u && asleep) atomicAdd(&w.ctr[C_ISL_SLEEPING], asleep);
    if (g.rank() == 0) {
        w.ctr[C_ISLANDS] = *(volatile uint32_t*)&st[IS_TOTAL];
        w.ctr[C_ISL_LARGEST] = *(volatile uint32_t*)&st[IS_LARGEST];
        if (w.ts) w.ts[TS_ISLANDS] = global_ns();
    }
    return g.sync();
}

template <class G>
__device__ bool phase_constraints(G& g, WorldDev& w, uint32_t cur, uint32_t* M_out, uint32_t* ncol_out,
                                  bool islands = true) {
    if (islands && !phase_islands(g, w, cur, w.scan)) return false;
    const uint32_t P = w.n_pairs, N = w.n_bodies;
    // 1. solver constraint list: manifolds that are not both-sleeping, pair order
    for (uint32_t p = g.rank(); p < P; p += g.size()) {
        const ManifoldRec& m = w.man[cur][p];
        uint32_t f = 0;
        if (m.n > 0u) {
            const PairInfo& pi = w.pinfo[p];
            const bool as = pi.ia != 0xFFFFFFFFu ? w.prop[pi.ia].sleeping != 0u : true;
            const bool bs = pi.ib != 0xFFFFFFFFu ? w.prop[pi.ib].sleeping != 0u : true;
            f = (as && bs) ? 0u : 1u;
        }
        w.flag[p] = f;
    }
    for (uint32_t i = g.rank(); i <= N; i += g.size()) {
        w.adj_off[i] = 0u;
        if (i < N) w.adj_cur[i] = 0u;
    }
    const uint32_t NG = w.cfg.owner_groups > 1u ? min(w.cfg.owner_groups, kMaxOwnerGroups) : 1u;
    for (uint32_t i = g.rank(); i < 257u; i += g.size()) {
        w.colour_cnt[i] = 0u;
        if (i < 256u) w.colour_cur[i] = 0u;
    }
    if (NG > 1u) {
        for (uint32_t i = g.rank(); i <= 256u * NG; i += g.size()) {
            w.ocnt[i] = 0u;
            if (i < 256u * NG) w.ocur[i] = 0u;
        }
        for (uint32_t i = g.rank(); i < 2u * kMaxOwnerGroups; i += g.size()) w.ocnt[kOwnerPoints + i] = 0u;
    }
    // colouring round counters (3) and position-sweep min separations (16)
    // live after the per-block scan partials
    if (g.rank() < 20u) w.scan[g.nblocks() + g.rank()] = 0u;
    if (!g.sync()) return false;
    uint32_t M = 0;
    if (!group_scan(
            g, P, [&](uint32_t i) { return w.flag[i]; },
            [&](uint32_t i, uint32_t pre) {
                if (w.flag[i]) w.cons[pre] = i;
            },
            w.scan, &M))
        return false;
    *M_out = M;
    uint32_t pts = 0;
    for (uint32_t k = g.rank(); k < M; k += g.size()) pts += w.man[cur][w.cons[k]].n;
    pts = warp_sum(pts);
    if ((threadIdx.x & 31) == 0 && pts) atomicAdd(&w.ctr[C_POINTS], pts);
    if (g.rank() == 0) w.ctr[C_CONSTRAINTS] = M;

    // 2. adjacency of the bodies the solver writes (dynamic, awake): the
    // constraints of each, for the colouring and for event-ordered sweeps
    uint32_t kin = 0;
    for (uint32_t k = g.rank(); k < M; k += g.size()) {
        const PairInfo& pi = w.pinfo[w.cons[k]];
        const DBodyProp& pa = w.prop[pi.ia];
        const DBodyProp& pb = w.prop[pi.ib];
        if (writable(pa)) atomicAdd(&w.adj_off[pi.ia], 1u);
        if (writable(pb)) atomicAdd(&w.adj_off[pi.ib], 1u);
        kin += ((pa.type == 1u && !pa.sleeping) || (pb.type == 1u && !pb.sleeping)) ? 1u : 0u;
    }
    kin = warp_sum(kin);
    if ((threadIdx.x & 31) == 0 && kin) atomicAdd(&w.ctr[C_KIN_CONTACT], kin);
    if (!g.sync()) return false;
    {
        uint32_t tot;
        // exclusive scan of the counts in place (group_scan reads and writes
        // each element in the same thread and tile); adj_cur is still zero
        if (!group_scan(
                g, N, [&](uint32_t i) { return w.adj_off[i]; }, [&](uint32_t i, uint32_t pre) { w.adj_off[i] = pre; },
                w.scan, &tot))
            return false;
        if (g.rank() == 0) w.adj_off[N] = tot;
        for (uint32_t k = g.rank(); k < M; k += g.size()) {
            const PairInfo& pi = w.pinfo[w.cons[k]];
            if (writable(w.prop[pi.ia])) w.adj[w.adj_off[pi.ia] + atomicAdd(&w.adj_cur[pi.ia], 1u)] = k;
            if (writable(w.prop[pi.ib])) w.adj[w.adj_off[pi.ib] + atomicAdd(&w.adj_cur[pi.ib], 1u)] = k;
            w.colour[k] = 0xFFFFFFFFu;
        }
        if (!g.sync()) return false;
    }

    // 3. colouring
    if (w.cfg.colouring == 1u) {
        // GraphColoring.build (islands.zig:668-736) over every manifold in
        // pair order, all bodies as nodes; one thread.
        for (uint32_t i = g.rank(); i < N * 8u; i += g.size()) w.bmask[i] = 0u;
        if (!g.sync()) return false;
        if (g.rank() == 0) {
            for (uint32_t p = 0; p < P; ++p) {
                const ManifoldRec& m = w.man[cur][p];
                if (m.n == 0u) continue;
                const PairInfo& pi = w.pinfo[p];
                uint32_t* ma = &w.bmask[pi.ia * 8u];
                uint32_t* mb = &w.bmask[pi.ib * 8u];
                uint32_t c = 0;
                while (c < 255u && (((ma[c >> 5] | mb[c >> 5]) >> (c & 31)) & 1u)) ++c;
                if (c == 255u) atomicOr(&w.ctr[C_ERROR], ERR_COLOURS);
                ma[c >> 5] |= 1u << (c & 31);
                mb[c >> 5] |= 1u << (c & 31);
                w.flag[p] = c;
            }
        }
        if (!g.sync()) return false;
        for (uint32_t k = g.rank(); k < M; k += g.size()) w.colour[k] = w.flag[w.cons[k]];
        if (!g.sync()) return false;
    } else {
        // Jones-Plassmann over writable bodies == greedy in priority order.
        // A manifold is coloured once every higher-priority neighbour is
        // (then no lower-priority one is yet).  On one CTA: rounds, a barrier
        // after each.  On several, no barrier: each thread polls its
        // manifolds until all are coloured (the highest-priority uncoloured
        // manifold can always be coloured by its thread, so this ends; the
        // wait is bounded by kColourTimeoutNs, ERR_TIMEOUT).
        const bool polling = g.nblocks() > 1u;
        const unsigned long long t_start = polling ? global_ns() : 0ull;
        // rounds: three rotating counters at scan[nblocks .. nblocks+3)
        uint32_t* rem = w.scan + g.nblocks();
        for (uint32_t round = 0;; ++round) {
            if (!polling && round > M + 1u) {
                if (g.rank() == 0) atomicOr(&w.ctr[C_ERROR], ERR_COLOURS);
                break;
            }
            if (!polling && g.rank() == 0) rem[(round + 1u) % 3u] = 0u;
            uint32_t left = 0;
            for (uint32_t k = g.rank(); k < M; k += g.size()) {
                volatile uint32_t* vc = w.colour;
                if (vc[k] != 0xFFFFFFFFu) continue;
                const PairInfo& pi = w.pinfo[w.cons[k]];
                uint32_t used[8] = {0, 0, 0, 0, 0, 0, 0, 0};
                bool ready = true;
                // both bodies' neighbours as one list (the bodies the solver
                // writes), their colours sixteen at a time, every load of a
                // batch issued before any is used (the colours were written
                // by other SMs in the last round: each load is a long one)
                const bool wa = writable(w.prop[pi.ia]), wb = writable(w.prop[pi.ib]);
                const uint32_t a0 = wa ? w.adj_off[pi.ia] : 0u, a1 = wa ? w.adj_off[pi.ia + 1u] : 0u;
                const uint32_t b0 = wb ? w.adj_off[pi.ib] : 0u, b1 = wb ? w.adj_off[pi.ib + 1u] : 0u;
                const uint32_t na = a1 - a0, nt = na + (b1 - b0);
                for (uint32_t t0 = 0; t0 < nt && ready; t0 += 16u) {
                    uint32_t jj[16], cc[16];
#pragma unroll
                    for (int q = 0; q < 16; ++q) {
                        const uint32_t t = t0 + (uint32_t)q;
                        jj[q] = t < nt ? w.adj[t < na ? a0 + t : b0 + (t - na)] : k;
                    }
#pragma unroll
                    for (int q = 0; q < 16; ++q) cc[q] = jj[q] != k ? vc[jj[q]] : 0xFFFFFFFEu;
#pragma unroll
                    for (int q = 0; q < 16; ++q) {
                        if (jj[q] == k) continue;
                        const uint32_t cj = cc[q];
                        if (cj == 0xFFFFFFFFu) {
                            if (jp_before(jj[q], k)) ready = false;
                        } else if (cj < 256u) {
                            used[cj >> 5] |= 1u << (cj & 31);
                        }
                    }
                }
                if (!ready) {
                    ++left;
                    continue;
                }
                uint32_t c = 256u;
                for (uint32_t wd = 0; wd < 8u; ++wd)
                    if (used[wd] != 0xFFFFFFFFu) {
                        c = wd * 32u + (uint32_t)(__ffs(~used[wd]) - 1);
                        break;
                    }
                if (c >= 256u) {
                    atomicOr(&w.ctr[C_ERROR], ERR_COLOURS);
                    c = 255u;
                }
                vc[k] = c;
            }
            if (polling) {
                if (left == 0u) break;
                if (global_ns() - t_start > kColourTimeoutNs) {
                    atomicOr(&w.ctr[C_ERROR], ERR_TIMEOUT);
                    break;
                }
                if ((*(volatile uint32_t*)&w.ctr[C_ERROR] & ERR_TIMEOUT) != 0u) break;
                continue;
            }
            left = warp_sum(left);
            if ((threadIdx.x & 31) == 0 && left) atomicAdd(&rem[round % 3u], left);
            if (!g.sync()) return false;
            const uint32_t r = *(volatile uint32_t*)&rem[round % 3u];
            if (r == 0u) break;
        }
        if (polling && !g.sync()) return false;
    }
    // 4. colour-major packing + ContactSolver.addManifold (solver.zig:449-491).
    // With owner groups, each colour is packed group by group: group =
    // home body mod NG, the home body being a if the solver writes it, else b
    // (the order inside a colour does not change any result).
    auto owner = [&](uint32_t k) -> uint32_t {
        const PairInfo& pi = w.pinfo[w.cons[k]];
        return (writable(w.prop[pi.ia]) ? pi.ia : pi.ib) % NG;
    };
    for (uint32_t k = g.rank(); k < M; k += g.size()) {
        if (w.colour[k] > 255u) w.colour[k] = 255u;  // only after ERR_COLOURS
        atomicAdd(&w.colour_cnt[w.colour[k]], 1u);
        if (NG > 1u) atomicAdd(&w.ocnt[w.colour[k] * NG + owner(k)], 1u);
    }
    if (!g.sync()) return false;
    if (NG > 1u && g.block() == 0u) {
        // exclusive scan of the (colour, group) counts, colour-major, by block
        // 0: each thread's run of at most 16 counts loaded at once (one round
        // trip, not one per count), scanned, stored
        constexpr uint32_t kPer = 16;
        const uint32_t E = 256u * NG, per = (E + blockDim.x - 1u) / blockDim.x, lo = threadIdx.x * per;
        uint32_t v[kPer];
        uint32_t sum = 0;
#pragma unroll
        for (uint32_t j = 0; j < kPer; ++j) {
            const uint32_t i = lo + j;
            v[j] = j < per && i < E ? w.ocnt[i] : 0u;
            sum += v[j];
        }
        // (blocks of fewer than 256 threads: the rest of each run one by one)
        for (uint32_t i = lo + kPer; i < min(E, lo + per); ++i) sum += w.ocnt[i];
        uint32_t total = 0;
        uint32_t run = block_excl_scan(sum, &total);
#pragma unroll
        for (uint32_t j = 0; j < kPer; ++j) {
            const uint32_t i = lo + j;
            if (j < per && i < E) {
                w.ocnt[i] = run;
                run += v[j];
            }
        }
        for (uint32_t i = lo + kPer; i < min(E, lo + per); ++i) {
            const uint32_t x = w.ocnt[i];
            w.ocnt[i] = run;
            run += x;
        }
        if (threadIdx.x == 0) w.ocnt[E] = total;
    }
    if (g.rank() < 32u) {
        // exclusive scan of the 256 colour counts by one warp: all eight
        // loads first, then the scans
        const uint32_t lane = threadIdx.x & 31;
        uint32_t v[8];
#pragma unroll
        for (uint32_t r = 0; r < 8u; ++r) v[r] = w.colour_cnt[32u * r + lane];
        uint32_t carry = 0, last = 0;
#pragma unroll
        for (uint32_t r = 0; r < 8u; ++r) {
            const uint32_t c0 = 32u * r;
            const uint32_t inc = warp_incl_scan(v[r]);
            const uint32_t nz = __ballot_sync(0xffffffffu, v[r] != 0u);
            if (nz) last = c0 + 32u - __clz(nz);
            w.colour_cnt[c0 + lane] = carry + inc - v[r];
            carry += __shfl_sync(0xffffffffu, inc, 31);
        }
        if (lane == 0) {
            w.colour_cnt[256] = carry;
            w.ctr[C_COLOURS] = last;
        }
    }
    if (!g.sync()) return false;
    *ncol_out = *(volatile uint32_t*)&w.ctr[C_COLOURS];
    for (uint32_t k = g.rank(); k < M; k += g.size()) {
        const uint32_t c = w.colour[k];
        uint32_t pos;
        if (NG > 1u) {
            const uint32_t o = owner(k), og = c * NG + o;
            pos = w.ocnt[og] + atomicAdd(&w.ocur[og], 1u);
            // points each sweep CTA would hold: by owner, and dealt round-robin
            const uint32_t np = w.man[cur][w.cons[k]].n;
            atomicAdd(&w.ocnt[kOwnerPoints + o], np);
            atomicAdd(&w.ocnt[kOwnerPoints + kMaxOwnerGroups + (pos - w.colour_cnt[c]) % NG], np);
        } else {
            pos = w.colour_cnt[c] + atomicAdd(&w.colour_cur[c], 1u);
        }
        const uint32_t p = w.cons[k];
        w.pos_of[k] = pos;
        w.packed_pair[pos] = p;
        const PairInfo& pi = w.pinfo[p];
        const ManifoldRec& m = w.man[cur][p];
        w.cm[pos] = make_uint4(pi.ia, pi.ib, m.n, p);
        w.cfr[pos] = make_float2(m.friction, m.restitution);
        const DBody& A = w.body[pi.ia];
        const DBody& B = w.body[pi.ib];
        const F3 pa = f3of(A.p), pb = f3of(B.p);
        const Qt qa = qof(A.q), qb = qof(B.q);
        for (uint32_t i = 0; i < m.n; ++i) {
            const ContactRec& ct = m.c[i];
            const F3 la{ct.la[0], ct.la[1], ct.la[2]}, lb{ct.lb[0], ct.lb[1], ct.lb[2]};
            const F3 nn{ct.normal[0], ct.normal[1], ct.normal[2]};
            const F3 wa = qrotate(qa, la) + pa;
            const F3 wb = qrotate(qb, lb) + pb;
            const F3 ad = wb - wa;
            const float base = -ct.penetration - dot3(ad, nn);
            const F3 ra = wa - pa, rb = wb - pb;
            float* cp = w.cp;
            cp[cpi(w, CP_NX, i, pos)] = nn.x; cp[cpi(w, CP_NY, i, pos)] = nn.y; cp[cpi(w, CP_NZ, i, pos)] = nn.z;
            cp[cpi(w, CP_LAX, i, pos)] = la.x; cp[cpi(w, CP_LAY, i, pos)] = la.y; cp[cpi(w, CP_LAZ, i, pos)] = la.z;
            cp[cpi(w, CP_LBX, i, pos)] = lb.x; cp[cpi(w, CP_LBY, i, pos)] = lb.y; cp[cpi(w, CP_LBZ, i, pos)] = lb.z;
            cp[cpi(w, CP_PX, i, pos)] = ct.point[0]; cp[cpi(w, CP_PY, i, pos)] = ct.point[1];
            cp[cpi(w, CP_PZ, i, pos)] = ct.point[2];
            cp[cpi(w, CP_RAX, i, pos)] = ra.x; cp[cpi(w, CP_RAY, i, pos)] = ra.y; cp[cpi(w, CP_RAZ, i, pos)] = ra.z;
            cp[cpi(w, CP_RBX, i, pos)] = rb.x; cp[cpi(w, CP_RBY, i, pos)] = rb.y; cp[cpi(w, CP_RBZ, i, pos)] = rb.z;
            cp[cpi(w, CP_BASE, i, pos)] = base;
            cp[cpi(w, CP_NM, i, pos)] = 0.f; cp[cpi(w, CP_TM0, i, pos)] = 0.f; cp[cpi(w, CP_TM1, i, pos)] = 0.f;
            cp[cpi(w, CP_T1X, i, pos)] = 0.f; cp[cpi(w, CP_T1Y, i, pos)] = 0.f; cp[cpi(w, CP_T1Z, i, pos)] = 0.f;
            cp[cpi(w, CP_T2X, i, pos)] = 0.f; cp[cpi(w, CP_T2Y, i, pos)] = 0.f; cp[cpi(w, CP_T2Z, i, pos)] = 0.f;
            cp[cpi(w, CP_BIAS, i, pos)] = 0.f;
            cp[cpi(w, CP_NI, i, pos)] = ct.normal_impulse;
            cp[cpi(w, CP_TI0, i, pos)] = ct.tangent_impulse[0];
            cp[cpi(w, CP_TI1, i, pos)] = ct.tangent_impulse[1];
        }
    }
    return g.sync();
}

// ---------------------------------------------------------------------------
// Solver building blocks (solver.zig:564-1005)
// ---------------------------------------------------------------------------
struct Soft {
    float bias_rate, mass_coeff, impulse_coeff;
};
__device__ __forceinline__ Soft soft_params(float hz, float zeta, float h) {  // solver.zig:57-72
    if (hz <= 0.0f) return Soft{0.f, 1.f, 1.f};
    const float pi = 3.14159274101257324f;
    const float omega = 2.0f * pi * hz;
    const float a1 = 2.0f * zeta + omega * h;
    const float a2 = h * omega * a1;
    const float a3 = 1.0f / (1.0f + a2);
    return Soft{omega / a1, a2 * a3, a3};
}
__device__ __forceinline__ F3 compute_orthogonal(F3 v) {  // solver.zig:967-981
    if (fabsf(v.x) < fabsf(v.y)) {
        if (fabsf(v.x) < fabsf(v.z)) return normalize_or_zero3(F3{0.f, -v.z, v.y});
        return normalize_or_zero3(F3{-v.y, v.x, 0.f});
    }
    if (fabsf(v.y) < fabsf(v.z)) return normalize_or_zero3(F3{-v.z, 0.f, v.x});
    return normalize_or_zero3(F3{-v.y, v.x, 0.f});
}
__device__ __forceinline__ Qt integrate_rotation_small(Qt r, F3 d) {  // solver.zig:984-1005
    const Qt h{d.x * 0.5f, d.y * 0.5f, d.z * 0.5f, 0.f};
    const Qt dq{h.w * r.x + h.x * r.w + h.y * r.z - h.z * r.y, h.w * r.y - h.x * r.z + h.y * r.w + h.z * r.x,
                h.w * r.z + h.x * r.y - h.y * r.x + h.z * r.w, h.w * r.w - h.x * r.x - h.y * r.y - h.z * r.z};
    return qnormalize(Qt{r.x + dq.x, r.y + dq.y, r.z + dq.z, r.w + dq.w});
}

// applyGravity for one dynamic awake body (solver.zig:564-605): gravity,
// extra damping below 0.5 m/s, damping, zeroing of tiny velocities.
__device__ __forceinline__ void body_gravity_d(float4& v4, float4& w4, float lin_damp, float ang_damp, F3 grav,
                                               float h) {
    F3 v = f3of(v4), av = f3of(w4);
    v = v + grav * h;
    float ld = lin_damp, adp = ang_damp;
    const float ls = len3(v), as = len3(av);
    if (ls < 0.5f) ld += 5.0f * (1.0f - (ls / 0.5f));
    if (as < 0.5f) adp += 5.0f * (1.0f - (as / 0.5f));
    const float ldec = fmaxf(0.0f, 1.0f - ld * h), adec = fmaxf(0.0f, 1.0f - adp * h);
    v = v * ldec;
    av = av * adec;
    if (lensq3(v) < 0.001f * 0.001f) v = F3{0.f, 0.f, 0.f};
    if (lensq3(av) < 0.001f * 0.001f) av = F3{0.f, 0.f, 0.f};
    v4 = make_float4(v.x, v.y, v.z, 0.f);
    w4 = make_float4(av.x, av.y, av.z, 0.f);
}
__device__ __forceinline__ void body_gravity(float4& v4, float4& w4, const DBodyProp& pr, F3 grav, float h) {
    body_gravity_d(v4, w4, pr.lin_damp, pr.ang_damp, grav, h);
}
// BodyState.integratePosition for one awake non-static body
// (solver.zig:341-356): position, rotation and, for dynamic bodies, the world
// inverse inertia.
__device__ __forceinline__ void body_integrate_il(DBody& b, const float* il_local, bool dynamic, float h,
                                                  bool disable_rotation) {
    const F3 x = f3of(b.p) + f3of(b.v) * h;
    Qt q = qof(b.q);
    if (!disable_rotation) q = integrate_rotation(q, f3of(b.w), h);
    b.p = make_float4(x.x, x.y, x.z, b.p.w);
    b.q = f4of(q);
    if (dynamic) {
        M33 il;
#pragma unroll
        for (int k = 0; k < 9; ++k) il.m[k] = il_local[k];
        const M33 m = world_inv_inertia(q, il);
        b.i0 = make_float4(m.m[0], m.m[1], m.m[2], 0.f);
        b.i1 = make_float4(m.m[3], m.m[4], m.m[5], 0.f);
        b.i2 = make_float4(m.m[6], m.m[7], m.m[8], 0.f);
    }
}
__device__ __forceinline__ void body_integrate(DBody& b, const DBodyProp& pr, float h, bool disable_rotation) {
    body_integrate_il(b, pr.il, pr.type == 2u, h, disable_rotation);
}

// Local copy of one body's velocity state for a manifold sweep.
struct BV {
    F3 p, v, w;
    float im;
    M33 I;
    bool wr;
};
__device__ __forceinline__ BV load_bv(const WorldDev& w, uint32_t i) {
    const DBody& b = w.body[i];
    BV r;
    const float4 p = b.p, v = b.v, ww = b.w, i0 = b.i0, i1 = b.i1, i2 = b.i2;
    r.p = f3of(p);
    r.im = p.w;
    r.v = f3of(v);
    r.w = f3of(ww);
    r.I.m[0] = i0.x; r.I.m[1] = i0.y; r.I.m[2] = i0.z;
    r.I.m[3] = i1.x; r.I.m[4] = i1.y; r.I.m[5] = i1.z;
    r.I.m[6] = i2.x; r.I.m[7] = i2.y; r.I.m[8] = i2.z;
    r.wr = writable(w.prop[i]);
    return r;
}
__device__ __forceinline__ F3 point_vel(const BV& b, F3 wp) { return b.v + cross3(b.w, wp - b.p); }
// A body the solver does not write keeps its velocities: selects, not a
// branch, so the compiler can interleave both bodies' updates (the sweeps'
// latency chain; 0.97 -> 0.94 ms for the cluster kernel on the pile).
__device__ __forceinline__ void apply_impulse(BV& b, F3 imp, F3 r) {  // BodyState.applyImpulseAtPoint
    const F3 v2 = b.v + imp * b.im;
    const F3 w2 = b.w + mat3_mul_vec(b.I, cross3(r, imp));
    b.v = F3{b.wr ? v2.x : b.v.x, b.wr ? v2.y : b.v.y, b.wr ? v2.z : b.v.z};
    b.w = F3{b.wr ? w2.x : b.w.x, b.wr ? w2.y : b.w.y, b.wr ? w2.z : b.w.z};
}
__device__ __forceinline__ void store_bv(WorldDev& w, uint32_t i, const BV& b) {
    if (!b.wr) return;
    w.body[i].v = make_float4(b.v.x, b.v.y, b.v.z, 0.f);
    w.body[i].w = make_float4(b.w.x, b.w.y, b.w.z, 0.f);
}
// The solver settings the per-point arithmetic reads, as values.
struct SolveFlags {
    bool friction, restitution;
    float slop, pos_rate, max_corr;
};
__device__ __forceinline__ SolveFlags solve_flags(const StepCfg& c) {
    return SolveFlags{c.friction_on != 0u, c.restitution_on != 0u, c.slop, c.pos_rate, c.max_pos_corr};
}

// The constraint-point fields of one manifold: field f of point s is
// b[f * sf + s * si].  In global memory b = cp + position, si = pair
// capacity, sf = 4 si; a chunk of the event-ordered sweeps held in shared
// memory has b = chunk + lane, si = 32, sf = 128; the cluster sweeps keep
// each point's fields together and a CTA's points one after another (b =
// rows + CP_NVEL x first point, sf = 1, si = CP_NVEL).
struct CPV {
    float* b;
    uint32_t sf, si;
};
__device__ __forceinline__ CPV cpv_global(const WorldDev& w, uint32_t pos) {
    return CPV{w.cp + pos, 4u * w.pair_cap, w.pair_cap};
}
__device__ __forceinline__ float& cpr(const CPV& v, uint32_t f, uint32_t s) {
    return v.b[(size_t)f * v.sf + (size_t)s * v.si];
}
__device__ __forceinline__ F3 ld3(const CPV& v, uint32_t f, uint32_t s) {
    return F3{cpr(v, f, s), cpr(v, f + 1, s), cpr(v, f + 2, s)};
}
__device__ __forceinline__ void st3(const CPV& v, uint32_t f, uint32_t s, F3 x) {
    cpr(v, f, s) = x.x;
    cpr(v, f + 1, s) = x.y;
    cpr(v, f + 2, s) = x.z;
}

// prepareConstraints for one point (solver.zig:608-699), from the two
// bodies' state after applyGravity.
// vin: the point's inputs (normal, local anchors, base separation); v: where
// its velocity-sweep fields go (the same rows, or a copy in shared memory).
// kTangents: v holds tangent2 too (else the sweeps recompute it as normal x
// tangent1, load_pt_row).
template <bool kTangents = true>
__device__ void prepare_point_s(const SolveFlags sf, const CPV vin, const CPV v, float restitution, uint32_t i,
                                const Soft& soft, float hinv, const BV& a, Qt qa, const BV& b, Qt qb) {
    const F3 n = ld3(vin, CP_NX, i);
    const F3 wa = qrotate(qa, ld3(vin, CP_LAX, i)) + a.p;
    const F3 wb = qrotate(qb, ld3(vin, CP_LBX, i)) + b.p;
    const F3 ra = wa - a.p, rb = wb - b.p;
    const F3 pt = (wa + wb) * 0.5f;
    const F3 ad = wb - wa;
    const float sep = cpr(vin, CP_BASE, i) + dot3(ad, n);
    const F3 rna = cross3(ra, n), rnb = cross3(rb, n);
    float k = a.im + b.im;
    k += dot3(rna, mat3_mul_vec(a.I, rna));
    k += dot3(rnb, mat3_mul_vec(b.I, rnb));
    const float nm = k > kEpsilon ? 1.0f / k : 0.0f;
    const F3 rv = point_vel(b, pt) - point_vel(a, pt);
    const float vn = dot3(rv, n);
    float bias;
    if (sep > 0.0f) bias = sep * hinv;
    else bias = fmaxf(soft.bias_rate * sep, -0.2f);
    if (sf.restitution && vn < -1.0f) bias = fmaxf(bias, -restitution * vn);
    st3(v, CP_RAX, i, ra);
    st3(v, CP_RBX, i, rb);
    st3(v, CP_PX, i, pt);
    cpr(v, CP_NM, i) = nm;
    cpr(v, CP_BIAS, i) = bias;
    if (sf.friction) {
        const F3 t1 = compute_orthogonal(n);
        const F3 t2 = cross3(n, t1);
        const F3 r1a = cross3(ra, t1), r1b = cross3(rb, t1);
        float k1 = a.im + b.im;
        k1 += dot3(r1a, mat3_mul_vec(a.I, r1a));
        k1 += dot3(r1b, mat3_mul_vec(b.I, r1b));
        const F3 r2a = cross3(ra, t2), r2b = cross3(rb, t2);
        float k2 = a.im + b.im;
        k2 += dot3(r2a, mat3_mul_vec(a.I, r2a));
        k2 += dot3(r2b, mat3_mul_vec(b.I, r2b));
        st3(v, CP_T1X, i, t1);
        if (kTangents) st3(v, CP_T2X, i, t2);
        cpr(v, CP_TM0, i) = k1 > kEpsilon ? 1.0f / k1 : 0.0f;
        cpr(v, CP_TM1, i) = k2 > kEpsilon ? 1.0f / k2 : 0.0f;
    }
}
__device__ void prepare_point(WorldDev& w, uint32_t pos, uint32_t i, const Soft& soft, float hinv) {
    const uint4 cmv = w.cm[pos];
    const BV a = load_bv(w, cmv.x), b = load_bv(w, cmv.y);
    const Qt qa = qof(w.body[cmv.x].q), qb = qof(w.body[cmv.y].q);
    const CPV v = cpv_global(w, pos);
    prepare_point_s(solve_flags(w.cfg), v, v, w.cfr[pos].y, i, soft, hinv, a, qa, b, qb);
}

// warmStart for one manifold (solver.zig:702-729), rows holding the tangents.
__device__ void warm_points(const CPV& v, uint32_t n, float scale, BV& a, BV& b) {
    for (uint32_t i = 0; i < n; ++i) {
        const float sn = cpr(v, CP_NI, i) * scale;
        const float s1 = cpr(v, CP_TI0, i) * scale;
        const float s2 = cpr(v, CP_TI1, i) * scale;
        const F3 nv = ld3(v, CP_NX, i);
        const F3 t1 = ld3(v, CP_T1X, i), t2 = ld3(v, CP_T2X, i);
        const F3 imp = (nv * sn + t1 * s1) + t2 * s2;
        apply_impulse(a, -imp, ld3(v, CP_RAX, i));
        apply_impulse(b, imp, ld3(v, CP_RBX, i));
        cpr(v, CP_NI, i) = sn;
        cpr(v, CP_TI0, i) = s1;
        cpr(v, CP_TI1, i) = s2;
    }
}
__device__ void warm_manifold(WorldDev& w, uint32_t pos, float scale) {
    const uint4 cmv = w.cm[pos];
    BV a = load_bv(w, cmv.x), b = load_bv(w, cmv.y);
    warm_points(cpv_global(w, pos), cmv.z, scale, a, b);
    store_bv(w, cmv.x, a);
    store_bv(w, cmv.y, b);
}

// The fields of one constraint point a velocity sweep reads.
struct PtV {
    F3 pt, n, ra, rb, t1, t2;
    float nm, bias, tm0, tm1, ni, ti0, ti1;
};
__device__ __forceinline__ PtV load_ptv(const CPV& v, uint32_t i) {
    PtV r;
    r.pt = ld3(v, CP_PX, i);
    r.n = ld3(v, CP_NX, i);
    r.ra = ld3(v, CP_RAX, i);
    r.rb = ld3(v, CP_RBX, i);
    r.t1 = ld3(v, CP_T1X, i);
    r.t2 = ld3(v, CP_T2X, i);
    r.nm = cpr(v, CP_NM, i);
    r.bias = cpr(v, CP_BIAS, i);
    r.tm0 = cpr(v, CP_TM0, i);
    r.tm1 = cpr(v, CP_TM1, i);
    r.ni = cpr(v, CP_NI, i);
    r.ti0 = cpr(v, CP_TI0, i);
    r.ti1 = cpr(v, CP_TI1, i);
    return r;
}

// solveVelocityConstraints + solveFriction for one manifold (solver.zig:732-838).
// Points run in slot order (Gauss-Seidel inside the manifold); the next
// point's fields are loaded before this point's results are stored, so the
// loads overlap the dependent arithmetic.
__device__ void velocity_points(const WorldDev& w, const CPV& v, uint32_t n, float fr, const Soft& soft,
                                bool use_bias, BV& a, BV& b) {
    if (n == 0u) return;
    PtV c = load_ptv(v, 0);
    for (uint32_t i = 0; i < n; ++i) {
        PtV nx;
        if (i + 1u < n) nx = load_ptv(v, i + 1u);
        const F3 rv = point_vel(b, c.pt) - point_vel(a, c.pt);
        const float vn = dot3(rv, c.n);
        float imp;
        if (use_bias)
            imp = -soft.mass_coeff * c.nm * (vn + c.bias) - soft.impulse_coeff * c.ni;
        else
            imp = -c.nm * vn;
        const float nn = fmaxf(c.ni + imp, 0.0f);
        imp = nn - c.ni;
        const float ni = nn;
        const F3 P = c.n * imp;
        apply_impulse(a, -P, c.ra);
        apply_impulse(b, P, c.rb);
        float ti0 = c.ti0, ti1 = c.ti1;
        if (w.cfg.friction_on && fr > 0.0f) {
            const float mf = fr * ni;
            {
                const F3 rv1 = point_vel(b, c.pt) - point_vel(a, c.pt);
                const float vt1 = dot3(rv1, c.t1);
                float f1 = -c.tm0 * vt1;
                const float o1 = ti0;
                ti0 = clampf_ref(o1 + f1, -mf, mf);
                f1 = ti0 - o1;
                const F3 I1 = c.t1 * f1;
                apply_impulse(a, -I1, c.ra);
                apply_impulse(b, I1, c.rb);
            }
            {
                const F3 rv2 = point_vel(b, c.pt) - point_vel(a, c.pt);
                const float vt2 = dot3(rv2, c.t2);
                float f2 = -c.tm1 * vt2;
                const float o2 = ti1;
                ti1 = clampf_ref(o2 + f2, -mf, mf);
                f2 = ti1 - o2;
                const F3 I2 = c.t2 * f2;
                apply_impulse(a, -I2, c.ra);
                apply_impulse(b, I2, c.rb);
            }
        }
        cpr(v, CP_NI, i) = ni;
        cpr(v, CP_TI0, i) = ti0;
        cpr(v, CP_TI1, i) = ti1;
        if (i + 1u < n) c = nx;
    }
}
// The same sweep without look-ahead: each point's fields are read when the
// point starts, which keeps fewer registers live (the event-ordered sweeps
// mostly read their rows from shared memory, where look-ahead gains little).
__device__ void velocity_points_near(bool friction, const CPV v, uint32_t n, float fr, const Soft& soft,
                                     bool use_bias, BV& a, BV& b) {
    for (uint32_t i = 0; i < n; ++i) {
        const PtV c = load_ptv(v, i);
        const F3 rv = point_vel(b, c.pt) - point_vel(a, c.pt);
        const float vn = dot3(rv, c.n);
        float imp;
        if (use_bias)
            imp = -soft.mass_coeff * c.nm * (vn + c.bias) - soft.impulse_coeff * c.ni;
        else
            imp = -c.nm * vn;
        const float nn = fmaxf(c.ni + imp, 0.0f);
        imp = nn - c.ni;
        const float ni = nn;
        const F3 P = c.n * imp;
        apply_impulse(a, -P, c.ra);
        apply_impulse(b, P, c.rb);
        float ti0 = c.ti0, ti1 = c.ti1;
        if (friction && fr > 0.0f) {
            const float mf = fr * ni;
            {
                const F3 rv1 = point_vel(b, c.pt) - point_vel(a, c.pt);
                const float vt1 = dot3(rv1, c.t1);
                float f1 = -c.tm0 * vt1;
                const float o1 = ti0;
                ti0 = clampf_ref(o1 + f1, -mf, mf);
                f1 = ti0 - o1;
                const F3 I1 = c.t1 * f1;
                apply_impulse(a, -I1, c.ra);
                apply_impulse(b, I1, c.rb);
            }
            {
                const F3 rv2 = point_vel(b, c.pt) - point_vel(a, c.pt);
                const float vt2 = dot3(rv2, c.t2);
                float f2 = -c.tm1 * vt2;
                const float o2 = ti1;
                ti1 = clampf_ref(o2 + f2, -mf, mf);
                f2 = ti1 - o2;
                const F3 I2 = c.t2 * f2;
                apply_impulse(a, -I2, c.ra);
                apply_impulse(b, I2, c.rb);
            }
        }
        cpr(v, CP_NI, i) = ni;
        cpr(v, CP_TI0, i) = ti0;
        cpr(v, CP_TI1, i) = ti1;
    }
}
// The velocity-sweep fields of one point held contiguously (CP_NVEL floats,
// 8-byte aligned, the cluster sweeps' rows in shared memory): eleven 8-byte
// loads from one base address instead of one load and one address per field.
static_assert(CP_NX == 0 && CP_PX == 3 && CP_RAX == 6 && CP_RBX == 9 && CP_T1X == 12 && CP_NM == 15 &&
                  CP_TM0 == 16 && CP_TM1 == 17 && CP_BIAS == 18 && CP_NI == 19 && CP_TI0 == 20 && CP_TI1 == 21 &&
                  CP_NVEL == 22,
              "contiguous point rows pair the fields as (NX NY) (NZ PX) (PY PZ) ... (TI0 TI1)");
__device__ __forceinline__ PtV load_pt_row(const float* r, bool friction) {
    const float2* q = reinterpret_cast<const float2*>(r);
    const float2 q0 = q[0], q1 = q[1], q2 = q[2], q3 = q[3], q4 = q[4], q5 = q[5], q6 = q[6], q7 = q[7], q8 = q[8],
                 q9 = q[9], q10 = q[10];
    PtV c;
    c.n = F3{q0.x, q0.y, q1.x};
    c.pt = F3{q1.y, q2.x, q2.y};
    c.ra = F3{q3.x, q3.y, q4.x};
    c.rb = F3{q4.y, q5.x, q5.y};
    // tangents as prepare leaves them: with friction, tangent1 =
    // computeOrthogonal(n) and tangent2 = n x tangent1; without, both zero as
    // the constraint table set them (the rows here never get tangent1)
    if (friction) {
        c.t1 = F3{q6.x, q6.y, q7.x};
        c.t2 = cross3(c.n, c.t1);
    } else {
        c.t1 = F3{0.f, 0.f, 0.f};
        c.t2 = F3{0.f, 0.f, 0.f};
    }
    c.nm = q7.y;
    c.tm0 = q8.x;
    c.tm1 = q8.y;
    c.bias = q9.x;
    c.ni = q9.y;
    c.ti0 = q10.x;
    c.ti1 = q10.y;
    return c;
}
// warm_points and velocity_points_near over contiguous point rows (rows =
// the manifold's first point); the same operations in the same order.
__device__ __forceinline__ void warm_points_rows(float* rows, uint32_t n, float scale, BV& a, BV& b,
                                                 bool friction) {
    for (uint32_t i = 0; i < n; ++i) {
        float* r = rows + (size_t)i * CP_NVEL;
        const PtV c = load_pt_row(r, friction);
        const float sn = c.ni * scale;
        const float s1 = c.ti0 * scale;
        const float s2 = c.ti1 * scale;
        const F3 imp = (c.n * sn + c.t1 * s1) + c.t2 * s2;
        apply_impulse(a, -imp, c.ra);
        apply_impulse(b, imp, c.rb);
        r[CP_NI] = sn;
        *reinterpret_cast<float2*>(r + CP_TI0) = make_float2(s1, s2);
    }
}
__device__ __forceinline__ void velocity_points_rows(bool friction, float* rows, uint32_t n, float fr,
                                                     const Soft& soft, bool use_bias, BV& a, BV& b) {
    for (uint32_t i = 0; i < n; ++i) {
        float* r = rows + (size_t)i * CP_NVEL;
        const PtV c = load_pt_row(r, friction);
        const F3 rv = point_vel(b, c.pt) - point_vel(a, c.pt);
        const float vn = dot3(rv, c.n);
        float imp;
        if (use_bias)
            imp = -soft.mass_coeff * c.nm * (vn + c.bias) - soft.impulse_coeff * c.ni;
        else
            imp = -c.nm * vn;
        const float nn = fmaxf(c.ni + imp, 0.0f);
        imp = nn - c.ni;
        const float ni = nn;
        const F3 P = c.n * imp;
        apply_impulse(a, -P, c.ra);
        apply_impulse(b, P, c.rb);
        float ti0 = c.ti0, ti1 = c.ti1;
        if (friction && fr > 0.0f) {
            const float mf = fr * ni;
            {
                const F3 rv1 = point_vel(b, c.pt) - point_vel(a, c.pt);
                const float vt1 = dot3(rv1, c.t1);
                float f1 = -c.tm0 * vt1;
                const float o1 = ti0;
                ti0 = clampf_ref(o1 + f1, -mf, mf);
                f1 = ti0 - o1;
                const F3 I1 = c.t1 * f1;
                apply_impulse(a, -I1, c.ra);
                apply_impulse(b, I1, c.rb);
            }
            {
                const F3 rv2 = point_vel(b, c.pt) - point_vel(a, c.pt);
                const float vt2 = dot3(rv2, c.t2);
                float f2 = -c.tm1 * vt2;
                const float o2 = ti1;
                ti1 = clampf_ref(o2 + f2, -mf, mf);
                f2 = ti1 - o2;
                const F3 I2 = c.t2 * f2;
                apply_impulse(a, -I2, c.ra);
                apply_impulse(b, I2, c.rb);
            }
        }
        r[CP_NI] = ni;
        *reinterpret_cast<float2*>(r + CP_TI0) = make_float2(ti0, ti1);
    }
}
__device__ void velocity_manifold(WorldDev& w, uint32_t pos, const Soft& soft, bool use_bias) {
    const uint4 cmv = w.cm[pos];
    if (cmv.z == 0u) return;
    const float fr = w.cfr[pos].x;
    BV a = load_bv(w, cmv.x), b = load_bv(w, cmv.y);
    velocity_points(w, cpv_global(w, pos), cmv.z, fr, soft, use_bias, a, b);
    store_bv(w, cmv.x, a);
    store_bv(w, cmv.y, b);
}

// One body's pose state for a position sweep.
struct PB {
    F3 x;
    Qt q;
    float im;
    M33 I;
    bool wr;
};
__device__ __forceinline__ PB pb_of(float4 p, float4 q, float4 i0, float4 i1, float4 i2, bool wr) {
    PB r;
    r.x = f3of(p);
    r.q = qof(q);
    r.im = p.w;
    r.I.m[0] = i0.x; r.I.m[1] = i0.y; r.I.m[2] = i0.z;
    r.I.m[3] = i1.x; r.I.m[4] = i1.y; r.I.m[5] = i1.z;
    r.I.m[6] = i2.x; r.I.m[7] = i2.y; r.I.m[8] = i2.z;
    r.wr = wr;
    return r;
}
__device__ __forceinline__ void store_pb(DBody* body, uint32_t i, const PB& b) {
    if (!b.wr) return;
    body[i].p = make_float4(b.x.x, b.x.y, b.x.z, b.im);
    body[i].q = f4of(b.q);
}

// solvePositionConstraints for one manifold (solver.zig:860-923).
__device__ void position_points(const SolveFlags sf, const CPV v, uint32_t n, PB& A, PB& B, float* min_sep,
                                float* max_pen) {
    F3 xa = A.x, xb = B.x;
    Qt qa = A.q, qb = B.q;
    const float ima = A.im, imb = B.im;
    const M33 Ia = A.I, Ib = B.I;
    const bool wa_ = A.wr, wb_ = B.wr;
    const float slop = sf.slop;
    for (uint32_t i = 0; i < n; ++i) {
        const F3 n = ld3(v, CP_NX, i);
        const F3 wa = qrotate(qa, ld3(v, CP_LAX, i)) + xa;
        const F3 wb = qrotate(qb, ld3(v, CP_LBX, i)) + xb;
        const F3 ad = wb - wa;
        const float sep = cpr(v, CP_BASE, i) + dot3(ad, n);
        *min_sep = fminf(*min_sep, sep);
        *max_pen = fmaxf(*max_pen, -sep);
        if (sep >= -slop) continue;
        const float corr = fmaxf(sf.pos_rate * (sep + slop), -sf.max_corr);
        const F3 ra = wa - xa, rb = wb - xb;
        const F3 rna = cross3(ra, n), rnb = cross3(rb, n);
        float k = ima + imb;
        k += dot3(rna, mat3_mul_vec(Ia, rna));
        k += dot3(rnb, mat3_mul_vec(Ib, rnb));
        if (k < kEpsilon) continue;
        const F3 pimp = n * (-corr / k);
        if (wa_) {
            xa = xa - pimp * ima;
            qa = integrate_rotation_small(qa, mat3_mul_vec(Ia, cross3(ra, -pimp)));
        }
        if (wb_) {
            xb = xb + pimp * imb;
            qb = integrate_rotation_small(qb, mat3_mul_vec(Ib, cross3(rb, pimp)));
        }
    }
    A.x = xa;
    A.q = qa;
    B.x = xb;
    B.q = qb;
}
// position_points over contiguous point rows that hold, once the velocity
// sweeps are done, each point's position-sweep inputs: the normal where the
// velocity rows keep it (CP_NX), local anchor a at CP_PX, local anchor b at
// CP_RAX, the base separation at CP_RBX.  The same operations in the same
// order.
__device__ void position_points_rows(const SolveFlags sf, const float* rows, uint32_t n, PB& A, PB& B,
                                     float* min_sep, float* max_pen) {
    F3 xa = A.x, xb = B.x;
    Qt qa = A.q, qb = B.q;
    const float ima = A.im, imb = B.im;
    const M33 Ia = A.I, Ib = B.I;
    const bool wa_ = A.wr, wb_ = B.wr;
    const float slop = sf.slop;
    for (uint32_t i = 0; i < n; ++i) {
        const float2* q = reinterpret_cast<const float2*>(rows + (size_t)i * CP_NVEL);
        const float2 q0 = q[0], q1 = q[1], q2 = q[2], q3 = q[3], q4 = q[4];
        const F3 n = F3{q0.x, q0.y, q1.x};
        const F3 la = F3{q1.y, q2.x, q2.y};
        const F3 lb = F3{q3.x, q3.y, q4.x};
        const float base = q4.y;
        const F3 wa = qrotate(qa, la) + xa;
        const F3 wb = qrotate(qb, lb) + xb;
        const F3 ad = wb - wa;
        const float sep = base + dot3(ad, n);
        *min_sep = fminf(*min_sep, sep);
        *max_pen = fmaxf(*max_pen, -sep);
        if (sep >= -slop) continue;
        const float corr = fmaxf(sf.pos_rate * (sep + slop), -sf.max_corr);
        const F3 ra = wa - xa, rb = wb - xb;
        const F3 rna = cross3(ra, n), rnb = cross3(rb, n);
        float k = ima + imb;
        k += dot3(rna, mat3_mul_vec(Ia, rna));
        k += dot3(rnb, mat3_mul_vec(Ib, rnb));
        if (k < kEpsilon) continue;
        const F3 pimp = n * (-corr / k);
        if (wa_) {
            xa = xa - pimp * ima;
            qa = integrate_rotation_small(qa, mat3_mul_vec(Ia, cross3(ra, -pimp)));
        }
        if (wb_) {
            xb = xb + pimp * imb;
            qb = integrate_rotation_small(qb, mat3_mul_vec(Ib, cross3(rb, pimp)));
        }
    }
    A.x = xa;
    A.q = qa;
    B.x = xb;
    B.q = qb;
}
static_assert(CP_NX == 0 && CP_PX == 3 && CP_RAX == 6 && CP_RBX == 9 && CP_NM > CP_RBX,
              "position rows: normal, anchor a, anchor b, base separation in the first ten floats");
__device__ void position_manifold(WorldDev& w, uint32_t pos, float* min_sep, float* max_pen) {
    const uint4 cmv = w.cm[pos];
    const DBodyProp& pa = w.prop[cmv.x];
    const DBodyProp& pb = w.prop[cmv.y];
    if (pa.type == 0u && pb.type == 0u) return;
    const DBody& A = w.body[cmv.x];
    const DBody& B = w.body[cmv.y];
    PB a = pb_of(A.p, A.q, A.i0, A.i1, A.i2, writable(pa));
    PB b = pb_of(B.p, B.q, B.i0, B.i1, B.i2, writable(pb));
    position_points(solve_flags(w.cfg), cpv_global(w, pos), cmv.z, a, b, min_sep, max_pen);
    store_pb(w.body, cmv.x, a);
    store_pb(w.body, cmv.y, b);
}

// End of one position sweep: reduce its min separation and max penetration
// over the group and decide the early break (solver.zig:917-921).
template <class G>
__device__ bool pos_sweep_end(G& g, WorldDev& w, uint32_t it, float mn, float mx, bool* brk) {
    int32_t kmn = fkey(mn), kmx = fkey(mx);
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        kmn = min(kmn, __shfl_xor_sync(0xffffffffu, kmn, d));
        kmx = max(kmx, __shfl_xor_sync(0xffffffffu, kmx, d));
    }
    int32_t* minsep = reinterpret_cast<int32_t*>(w.scan + g.nblocks() + 4u);  // 16 slots
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&minsep[it & 15u], kmn);
        atomicMax(reinterpret_cast<int32_t*>(&w.ctr[C_MAX_PEN_KEY]), kmx);
    }
    if (g.rank() == 0) w.ctr[C_POS_ITERS] += 1u;
    if (!g.sync()) return false;
    const float ms = fkey_inv(*(volatile int32_t*)&minsep[it & 15u]);
    *brk = ms >= -3.0f * w.cfg.slop;
    return true;
}

// ---------------------------------------------------------------------------
// Phase: solve (ContactSolver.solve, solver.zig:494-561)
// ---------------------------------------------------------------------------
template <class G>
__device__ bool phase_solve(G& g, WorldDev& w, uint32_t M, uint32_t ncol) {
    const StepCfg& cf = w.cfg;
    const float dt = cf.dt;
    const bool has = M > 0u;
    const float h = dt / (float)cf.substeps;
    const Soft soft = soft_params(cf.hertz, cf.damping_ratio, h);
    const float hinv = h > kEpsilon ? 1.0f / h : 0.0f;
    const Soft hard{0.f, 1.f, 1.f};
    const F3 grav{cf.gravity[0], cf.gravity[1], cf.gravity[2]};
    const uint32_t N = w.n_bodies;
    for (uint32_t s = 0; s < cf.substeps; ++s) {
        // applyGravity (solver.zig:564-605)
        for (uint32_t i = g.rank(); i < N; i += g.size()) {
            const DBodyProp& pr = w.prop[i];
            if (!(pr.type == 2u && pr.sleeping == 0u)) continue;
            DBody& b = w.body[i];
            float4 v = b.v, av = b.w;
            body_gravity(v, av, pr, grav, h);
            b.v = v;
            b.w = av;
        }
        if (!g.sync()) return false;
        if (has) {
            for (uint32_t it = g.rank(); it < 4u * M; it += g.size()) {
                const uint32_t slot = it / M, pos = it - slot * M;
                if (slot < w.cm[pos].z) prepare_point(w, pos, slot, soft, hinv);
            }
            if (!g.sync()) return false;
            if (cf.warm_starting && s == 0u) {
                for (uint32_t c = 0; c < ncol; ++c) {
                    const uint32_t lo = w.colour_cnt[c], hi = w.colour_cnt[c + 1u];
                    for (uint32_t pos = lo + g.rank(); pos < hi; pos += g.size()) warm_manifold(w, pos, cf.warm_scale);
                    if (!g.sync()) return false;
                }
            }
            for (uint32_t vi = 0; vi < cf.vel_iters; ++vi) {
                for (uint32_t c = 0; c < ncol; ++c) {
                    const uint32_t lo = w.colour_cnt[c], hi = w.colour_cnt[c + 1u];
                    for (uint32_t pos = lo + g.rank(); pos < hi; pos += g.size()) velocity_manifold(w, pos, soft, true);
                    if (!g.sync()) return false;
                }
            }
        }
        // integratePositions (solver.zig:841-845, 341-356)
        for (uint32_t i = g.rank(); i < N; i += g.size()) {
            const DBodyProp& pr = w.prop[i];
            if (pr.type == 0u || pr.sleeping) continue;
            DBody b = w.body[i];
            body_integrate(b, pr, h, cf.disable_rotation != 0u);
            w.body[i] = b;
        }
        if (!g.sync()) return false;
        if (has) {
            for (uint32_t c = 0; c < ncol; ++c) {
                const uint32_t lo = w.colour_cnt[c], hi = w.colour_cnt[c + 1u];
                for (uint32_t pos = lo + g.rank(); pos < hi; pos += g.size()) velocity_manifold(w, pos, hard, false);
                if (!g.sync()) return false;
            }
        }
        // test hook: every body's state after this substep (the thread that
        // records body i also applies its next gravity step)
        if (cf.record_substeps && w.subrec) {
            for (uint32_t i = g.rank(); i < N; i += g.size()) {
                const DBody b = w.body[i];
                float* r = w.subrec + ((size_t)s * N + i) * 13u;
                r[0] = b.p.x; r[1] = b.p.y; r[2] = b.p.z;
                r[3] = b.q.x; r[4] = b.q.y; r[5] = b.q.z; r[6] = b.q.w;
                r[7] = b.v.x; r[8] = b.v.y; r[9] = b.v.z;
                r[10] = b.w.x; r[11] = b.w.y; r[12] = b.w.z;
            }
            if (g.rank() == 0) w.ctr[C_SUBREC] = s + 1u;
        }
    }
    if (has) {
        for (uint32_t it = 0; it < cf.pos_iters; ++it) {
            float mn = 0.0f, mx = -__int_as_float(0x7f800000);
            for (uint32_t c = 0; c < ncol; ++c) {
                const uint32_t lo = w.colour_cnt[c], hi = w.colour_cnt[c + 1u];
                for (uint32_t pos = lo + g.rank(); pos < hi; pos += g.size()) position_manifold(w, pos, &mn, &mx);
                if (!g.sync()) return false;
            }
            bool brk = false;
            if (!pos_sweep_end(g, w, it, mn, mx, &brk)) return false;
            if (brk) break;
        }
    }
    return true;
}

// ---------------------------------------------------------------------------
// Phase: solve with event-ordered sweeps
// ---------------------------------------------------------------------------
// Every sweep of ContactSolver.solve visits the manifolds in colour-major
// order, and a manifold reads and writes only its two bodies.  The result of
// the sweeps is therefore fixed by the order in which each body sees its own
// manifolds: in sweep k, body b (d_b manifolds) sees them in position order as
// events k*d_b .. k*d_b + d_b - 1.  Here each manifold waits until every body
// it writes has seen exactly the events before its own (one counter per
// body), applies itself and advances those counters.  Nothing waits for a
// whole colour batch or a whole sweep: a manifold of the next sweep starts as
// soon as its own bodies are through.  The body steps between sweeps are done
// by the manifold that applies a body's last event of the sweep before them
// (integrate after the last velocity sweep of a substep, gravity after the
// relax sweep), and prepare reads a copy of each body taken right after its
// gravity step.  Each body sees the same operations in the same order as with
// a barrier after every colour batch, so the results are bit-identical.
//
// Progress: a warp takes its chunks in increasing (sweep, chunk) order, the
// chunks are colour-major and a chunk only waits for chunks earlier in that
// order (a chunk's manifolds share no written body), so the earliest
// unfinished chunk of the whole group is always ready; all blocks of a group
// are resident.  Every wait is bounded (kFlowTimeoutNs) and ends the step with
// ERR_TIMEOUT, which also stops every other waiting warp.  A step whose
// colouring overflowed (ERR_COLOURS: one colour may then hold manifolds of
// the same body) uses colour barriers instead.
constexpr unsigned long long kFlowTimeoutNs = 2000000000ull;

enum : uint32_t { FK_WARM = 0, FK_VEL = 1, FK_RELAX = 2, FK_POS = 3 };
struct FlowSweep {
    uint32_t kind, s, r;  // kind, substep, velocity iteration (FK_VEL) or position iteration (FK_POS)
};
// Floats of one chunk's constraint-point fields in shared memory.
constexpr uint32_t kChunkFloats = CP_NFIELDS * 4u * 32u;
// Everything the per-manifold steps read besides their own rows, passed by
// value so that none of it is re-read from memory between points.
struct FlowCtx {
    uint32_t W, S, V;  // warm-start sweep (0/1), substeps, velocity iterations
    uint32_t smem_chunks;  // chunks of each block held in shared memory
    Soft soft, hard;
    float h, hinv, warm_scale;
    F3 grav;
    bool dis_rot;
    SolveFlags sf;
    DBody* body;
    DBody* snap;
    const DBodyProp* prop;
    const float2* cfr;
    uint32_t n_bodies;
};
__device__ __forceinline__ FlowSweep flow_sweep(uint32_t k, const FlowCtx& fc) {
    if (fc.W) {
        if (k == 0u) return FlowSweep{FK_WARM, 0u, 0u};
        k -= 1u;
    }
    const uint32_t per = fc.V + 1u;
    if (k < fc.S * per) {
        const uint32_t s = k / per, r = k - s * per;
        return FlowSweep{r < fc.V ? FK_VEL : FK_RELAX, s, r};
    }
    return FlowSweep{FK_POS, fc.S, k - fc.S * per};
}

__device__ __forceinline__ uint32_t ld_relaxed_u32(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed_u32(uint32_t* p, uint32_t v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void fence_acq_rel_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

// A body record read through L2: another SM may have written it this step.
__device__ __forceinline__ DBody ld_body_cg(const DBody* b) {
    const float4* f = reinterpret_cast<const float4*>(b);
    DBody r;
    r.p = __ldcg(f + 0);
    r.q = __ldcg(f + 1);
    r.v = __ldcg(f + 2);
    r.w = __ldcg(f + 3);
    r.i0 = __ldcg(f + 4);
    r.i1 = __ldcg(f + 5);
    r.i2 = __ldcg(f + 6);
    return r;
}
__device__ __forceinline__ BV bv_of(const DBody& d, bool wr) {
    BV r;
    r.p = f3of(d.p);
    r.im = d.p.w;
    r.v = f3of(d.v);
    r.w = f3of(d.w);
    r.I.m[0] = d.i0.x; r.I.m[1] = d.i0.y; r.I.m[2] = d.i0.z;
    r.I.m[3] = d.i1.x; r.I.m[4] = d.i1.y; r.I.m[5] = d.i1.z;
    r.I.m[6] = d.i2.x; r.I.m[7] = d.i2.y; r.I.m[8] = d.i2.z;
    r.wr = wr;
    return r;
}

// Writes one body back after a velocity-type sweep event, with the body step
// that follows its last event of the sweep.
// The body step after a body's last event of sweep sw: 1 integrate, 2 gravity.
__device__ __forceinline__ uint32_t flow_body_op(const FlowCtx& fc, const FlowSweep& sw, uint32_t rank, uint32_t deg) {
    if (rank == 0xFFFFFFFFu || rank + 1u != deg) return 0u;
    if (sw.kind == FK_VEL && sw.r + 1u == fc.V) return 1u;
    if (sw.kind == FK_RELAX && sw.s + 1u < fc.S) return 2u;
    return 0u;
}
// The body properties that body step reads (op 1: local inverse inertia,
// op 2: the two damping coefficients), asked into L1 ahead of use ...
__device__ __forceinline__ void flow_prefetch_prop(const FlowCtx& fc, uint32_t op, uint32_t i) {
    if (op == 0u) return;
    const char* p = reinterpret_cast<const char*>(fc.prop + i);
    asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
    asm volatile("prefetch.global.L1 [%0];" ::"l"(p + sizeof(DBodyProp) - 1));
}
// ... and read when the step runs.
__device__ __forceinline__ void flow_ld_prop(const FlowCtx& fc, uint32_t op, uint32_t i, float pr[9]) {
    if (op == 1u) {
#pragma unroll
        for (int k = 0; k < 9; ++k) pr[k] = fc.prop[i].il[k];
    } else if (op == 2u) {
        pr[0] = fc.prop[i].lin_damp;
        pr[1] = fc.prop[i].ang_damp;
    }
}
// Writes one body back after a velocity-type sweep event, with the body step
// that follows its last event of the sweep.
__device__ __forceinline__ void flow_body_out(const FlowCtx& fc, uint32_t op, uint32_t i, const BV& x, Qt q,
                                              const float pr[9], uint32_t snap_par) {
    const float4 v4 = make_float4(x.v.x, x.v.y, x.v.z, 0.f), w4 = make_float4(x.w.x, x.w.y, x.w.z, 0.f);
    if (op == 0u) {
        fc.body[i].v = v4;
        fc.body[i].w = w4;
        return;
    }
    DBody d;
    d.p = make_float4(x.p.x, x.p.y, x.p.z, x.im);
    d.q = f4of(q);
    d.v = v4;
    d.w = w4;
    d.i0 = make_float4(x.I.m[0], x.I.m[1], x.I.m[2], 0.f);
    d.i1 = make_float4(x.I.m[3], x.I.m[4], x.I.m[5], 0.f);
    d.i2 = make_float4(x.I.m[6], x.I.m[7], x.I.m[8], 0.f);
    if (op == 1u) {
        body_integrate_il(d, pr, true, fc.h, fc.dis_rot);  // integratePositions of substep s
        fc.body[i] = d;
    } else {
        body_gravity_d(d.v, d.w, pr[0], pr[1], fc.grav, fc.h);  // applyGravity of substep s + 1
        fc.body[i].v = d.v;
        fc.body[i].w = d.w;
        fc.snap[(size_t)snap_par * fc.n_bodies + i] = d;
    }
}

// prepareConstraints of substep s for one manifold, from its bodies' state
// right after applyGravity of that substep (the copy in w.snap for bodies the
// solver writes; the others do not change during the solve).
__device__ __noinline__ void flow_prepare(const FlowCtx fc, uint32_t s, uint32_t pos, const CPV v, const uint4 cmv,
                                          const uint4 rkv) {
    if (cmv.z == 0u) return;
    const bool wa = rkv.x != 0xFFFFFFFFu, wb = rkv.z != 0xFFFFFFFFu;
    const size_t so = (size_t)(s & 1u) * fc.n_bodies;
    const DBody SA = ld_body_cg((wa ? fc.snap + so : fc.body) + cmv.x);
    const DBody SB = ld_body_cg((wb ? fc.snap + so : fc.body) + cmv.y);
    const BV sa = bv_of(SA, wa), sb = bv_of(SB, wb);
    const float rest = fc.cfr[pos].y;
    for (uint32_t i = 0; i < cmv.z; ++i)
        prepare_point_s(fc.sf, v, v, rest, i, fc.soft, fc.hinv, sa, qof(SA.q), sb, qof(SB.q));
}

// One manifold in one sweep, once its bodies are ready.
__device__ __noinline__ void flow_item(const FlowCtx fc, uint32_t k, uint32_t pos, const CPV v, const uint4 cmv,
                                       const uint4 rkv, float* mn, float* mx) {
    const FlowSweep sw = flow_sweep(k, fc);
    const bool wa = rkv.x != 0xFFFFFFFFu, wb = rkv.z != 0xFFFFFFFFu;
    if (sw.kind == FK_POS) {
        if (!wa && !wb && fc.prop[cmv.x].type == 0u && fc.prop[cmv.y].type == 0u) return;
        const DBody A = ld_body_cg(fc.body + cmv.x), B = ld_body_cg(fc.body + cmv.y);
        PB a = pb_of(A.p, A.q, A.i0, A.i1, A.i2, wa), b = pb_of(B.p, B.q, B.i0, B.i1, B.i2, wb);
        position_points(fc.sf, v, cmv.z, a, b, mn, mx);
        store_pb(fc.body, cmv.x, a);
        store_pb(fc.body, cmv.y, b);
        return;
    }
    const uint32_t opa = flow_body_op(fc, sw, rkv.x, rkv.y), opb = flow_body_op(fc, sw, rkv.z, rkv.w);
    flow_prefetch_prop(fc, opa, cmv.x);
    flow_prefetch_prop(fc, opb, cmv.y);
    Qt qa, qb;
    BV a, b;
    {
        const DBody A = ld_body_cg(fc.body + cmv.x), B = ld_body_cg(fc.body + cmv.y);
        a = bv_of(A, wa);
        b = bv_of(B, wb);
        qa = qof(A.q);
        qb = qof(B.q);
    }
    const float fr = fc.cfr[pos].x;
    if (sw.kind == FK_WARM)
        warm_points(v, cmv.z, fc.warm_scale, a, b);
    else
        velocity_points_near(fc.sf.friction, v, cmv.z, fr, sw.kind == FK_VEL ? fc.soft : fc.hard, sw.kind == FK_VEL, a, b);
    const uint32_t par = (sw.s + 1u) & 1u;
    float pr[9];
    if (wa) {
        flow_ld_prop(fc, opa, cmv.x, pr);
        flow_body_out(fc, opa, cmv.x, a, qa, pr, par);
    }
    if (wb) {
        flow_ld_prop(fc, opb, cmv.y, pr);
        flow_body_out(fc, opb, cmv.y, b, qb, pr, par);
    }
}

// Waits until every lane of the warp sees its bodies' event counters at the
// values given (at_least: at or past them).  Bounded: gives up after
// kFlowTimeoutNs or when another warp gave up, returning false.
__device__ __forceinline__ bool flow_wait(WorldDev& w, bool need_a, uint32_t a, uint32_t ea, bool need_b, uint32_t b,
                                          uint32_t eb, bool at_least) {
    bool ready = !need_a && !need_b;
    uint32_t spins = 0;
    unsigned long long t0 = 0;
    while (true) {
        if (!ready) {
            const uint32_t va = need_a ? ld_relaxed_u32(w.ev + a) : ea;
            const uint32_t vb = need_b ? ld_relaxed_u32(w.ev + b) : eb;
            ready = at_least ? (va >= ea && vb >= eb) : (va == ea && vb == eb);
        }
        if (__all_sync(0xffffffffu, ready)) return true;
        if (spins == 0u) t0 = global_ns();
        ++spins;
        bool stop = false;
        if ((spins & 63u) == 0u) {
            if (global_ns() - t0 > kFlowTimeoutNs) atomicOr(&w.ctr[C_ERROR], ERR_TIMEOUT);
            stop = (ld_relaxed_u32(&w.ctr[C_ERROR]) & ERR_TIMEOUT) != 0u;
        }
        if (__any_sync(0xffffffffu, stop)) return false;
        __nanosleep(20);
    }
}

// Runs sweeps [k0, k1).  The packed manifolds are cut into chunks of at most
// 32 positions that never cross a colour boundary (w.chunk: first and end
// position), so the manifolds of one chunk share no body the solver writes.
// Warp gw of the group takes chunks gw, gw + nwarps, ... in every sweep; it
// waits until all 32 lanes' bodies are ready, then the whole warp applies its
// chunk at once.  Warps are numbered across blocks first, spreading the
// chunks of a sweep over as many SMs as the group has.  Block b's L-th chunk
// is chunk L * nblocks + b; the first fc.smem_chunks of them keep their
// constraint-point fields in shared memory (fsm) for the whole solve.
template <class G>
__device__ bool flow_run(G& g, WorldDev& w, const FlowCtx& fc, float* fsm, uint32_t T, uint32_t k0, uint32_t k1,
                         float* mn, float* mx) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nwb = blockDim.x >> 5;
    const uint32_t gw = (threadIdx.x >> 5) * g.nblocks() + g.block(), nw = nwb * g.nblocks();
    const uint32_t nj = gw < T ? (T - gw + nw - 1u) / nw : 0u;
    if (nj == 0u) return true;  // uniform over the warp
    for (uint32_t k = k0; k < k1; ++k) {
        const FlowSweep sw = flow_sweep(k, fc);
        const bool first = sw.kind == FK_WARM || (sw.kind == FK_VEL && sw.r == 0u && !(fc.W && sw.s == 0u));
        for (uint32_t j = 0; j < nj; ++j) {
            const uint2 ch = w.chunk[gw + j * nw];
            const uint32_t pos = ch.x + lane;
            bool valid = pos < ch.y && ch.y <= w.pair_cap;
            const uint32_t L = (threadIdx.x >> 5) + j * nwb;
            const CPV v =
                L < fc.smem_chunks ? CPV{fsm + (size_t)L * kChunkFloats + lane, 128u, 32u} : cpv_global(w, pos);
            uint4 cmv = make_uint4(0u, 0u, 0u, 0u), rkv = make_uint4(0xFFFFFFFFu, 0u, 0xFFFFFFFFu, 0u);
            if (valid) {
                cmv = w.cm[pos];
                rkv = w.rk[pos];
                // guard: an index out of range is reported, never followed
                if (cmv.x >= w.n_bodies || cmv.y >= w.n_bodies || cmv.z > 4u ||
                    (rkv.x != 0xFFFFFFFFu && rkv.x >= rkv.y) || (rkv.z != 0xFFFFFFFFu && rkv.z >= rkv.w)) {
                    atomicOr(&w.ctr[C_ERROR], ERR_BOUNDS);
                    valid = false;
                    cmv = make_uint4(0u, 0u, 0u, 0u);
                    rkv = make_uint4(0xFFFFFFFFu, 0u, 0xFFFFFFFFu, 0u);
                }
            }
            const bool need_a = rkv.x != 0xFFFFFFFFu, need_b = rkv.z != 0xFFFFFFFFu;
            if (first) {
                // first sweep of a substep: prepare as soon as both bodies are
                // through the previous sweep (their gravity copy is written),
                // ahead of this manifold's own turn in the sweep
                if (!flow_wait(w, need_a, cmv.x, k * rkv.y, need_b, cmv.y, k * rkv.w, true)) return false;
                fence_acq_rel_gpu();
                if (valid) flow_prepare(fc, sw.s, pos, v, cmv, rkv);
            }
            const uint32_t ea = k * rkv.y + rkv.x, eb = k * rkv.w + rkv.z;
            if (!flow_wait(w, need_a, cmv.x, ea, need_b, cmv.y, eb, false)) return false;
            fence_acq_rel_gpu();
            if (valid) flow_item(fc, k, pos, v, cmv, rkv, mn, mx);
            fence_acq_rel_gpu();
            if (need_a) st_relaxed_u32(w.ev + cmv.x, ea + 1u);
            if (need_b) st_relaxed_u32(w.ev + cmv.y, eb + 1u);
        }
    }
    return true;
}

template <class G>
__device__ bool phase_solve_flow(G& g, WorldDev& w, float* fsm, uint32_t M, uint32_t ncol) {
    const StepCfg& cf = w.cfg;
    FlowCtx fc;
    fc.S = cf.substeps;
    fc.V = cf.vel_iters;
    fc.W = (cf.warm_starting && M > 0u) ? 1u : 0u;
    fc.h = cf.dt / (float)cf.substeps;
    fc.soft = soft_params(cf.hertz, cf.damping_ratio, fc.h);
    fc.hard = Soft{0.f, 1.f, 1.f};
    fc.hinv = fc.h > kEpsilon ? 1.0f / fc.h : 0.0f;
    fc.warm_scale = cf.warm_scale;
    fc.grav = F3{cf.gravity[0], cf.gravity[1], cf.gravity[2]};
    fc.dis_rot = cf.disable_rotation != 0u;
    fc.smem_chunks = cf.flow_smem_chunks;
    fc.sf = solve_flags(cf);
    fc.body = w.body;
    fc.snap = w.snap;
    fc.prop = w.prop;
    fc.cfr = w.cfr;
    fc.n_bodies = w.n_bodies;
    const uint32_t N = w.n_bodies;
    // Bodies: counters to zero; gravity of substep 0 and its copy for
    // prepare; a moving body without constraints takes all its substeps now.
    for (uint32_t i = g.rank(); i < N; i += g.size()) {
        w.ev[i] = 0u;
        const DBodyProp& pr = w.prop[i];
        const bool dyn = pr.type == 2u && !pr.sleeping, kin = pr.type == 1u && !pr.sleeping;
        if (!dyn && !kin) continue;
        DBody b = w.body[i];
        const uint32_t deg = dyn ? w.adj_off[i + 1u] - w.adj_off[i] : 0u;
        if (deg == 0u) {
            for (uint32_t s = 0; s < fc.S; ++s) {
                if (dyn) body_gravity(b.v, b.w, pr, fc.grav, fc.h);
                body_integrate(b, pr, fc.h, fc.dis_rot);
            }
        } else {
            body_gravity(b.v, b.w, pr, fc.grav, fc.h);
            w.snap[i] = b;
        }
        w.body[i] = b;
    }
    // Manifolds: rank among the constraints of each writable body, in
    // position order, and that body's constraint count.
    for (uint32_t k = g.rank(); k < M; k += g.size()) {
        const uint32_t pos = w.pos_of[k];
        const uint4 cmv = w.cm[pos];
        uint32_t r[2] = {0xFFFFFFFFu, 0xFFFFFFFFu}, d[2] = {0u, 0u};
        const uint32_t bodies[2] = {cmv.x, cmv.y};
        for (int t = 0; t < 2; ++t) {
            const uint32_t bi = bodies[t];
            if (!writable(w.prop[bi])) continue;
            const uint32_t lo = w.adj_off[bi], hi = w.adj_off[bi + 1u];
            uint32_t c = 0;
            for (uint32_t e = lo; e < hi; ++e) c += w.pos_of[w.adj[e]] < pos ? 1u : 0u;
            r[t] = c;
            d[t] = hi - lo;
        }
        w.rk[pos] = make_uint4(r[0], d[0], r[1], d[1]);
    }
    // Chunks: colour c's positions [colour_cnt[c], colour_cnt[c + 1]) in
    // pieces of 32, colour-major.
    uint32_t T = 0;
    for (uint32_t c = 0; c < ncol; ++c) {
        const uint32_t lo = w.colour_cnt[c], hi = w.colour_cnt[c + 1u];
        const uint32_t nch = (hi - lo + 31u) >> 5;
        for (uint32_t i = g.rank(); i < nch; i += g.size())
            w.chunk[T + i] = make_uint2(lo + 32u * i, min(lo + 32u * i + 32u, hi));
        T += nch;
    }
    if (!g.sync()) return false;
    if (M == 0u) return true;
    // this block's shared-memory chunks: fields from the packed arrays
    const uint32_t nb = g.nblocks(), blk = g.block();
    for (uint32_t L = 0; L < fc.smem_chunks && L * nb + blk < T; ++L) {
        const uint2 ch = w.chunk[L * nb + blk];
        for (uint32_t e = threadIdx.x; e < CP_NFIELDS * 4u * 32u; e += blockDim.x) {
            const uint32_t fs = e >> 5, ln = e & 31u;
            fsm[(size_t)L * kChunkFloats + e] = ch.x + ln < ch.y ? w.cp[(size_t)fs * w.pair_cap + ch.x + ln] : 0.0f;
        }
    }
    __syncthreads();
    const uint32_t K0 = fc.W + fc.S * (fc.V + 1u);
    float mn = 0.0f, mx = -__int_as_float(0x7f800000);
    if (!flow_run(g, w, fc, fsm, T, 0u, K0 + (cf.pos_iters ? 1u : 0u), &mn, &mx)) return false;
    for (uint32_t it = 0; it < cf.pos_iters; ++it) {
        if (it > 0u) {
            mn = 0.0f;
            mx = -__int_as_float(0x7f800000);
            if (!flow_run(g, w, fc, fsm, T, K0 + it, K0 + it + 1u, &mn, &mx)) return false;
        }
        bool brk = false;
        if (!pos_sweep_end(g, w, it, mn, mx, &brk)) return false;
        if (brk) break;
    }
    // impulses and masses back to the packed arrays (storeImpulses reads them)
    __syncthreads();
    const uint32_t back[6] = {CP_NM, CP_TM0, CP_TM1, CP_NI, CP_TI0, CP_TI1};
    for (uint32_t L = 0; L < fc.smem_chunks && L * nb + blk < T; ++L) {
        const uint2 ch = w.chunk[L * nb + blk];
        for (uint32_t e = threadIdx.x; e < 6u * 4u * 32u; e += blockDim.x) {
            const uint32_t fs = back[e >> 7] * 4u + ((e >> 5) & 3u), ln = e & 31u;
            if (ch.x + ln < ch.y) w.cp[(size_t)fs * w.pair_cap + ch.x + ln] = fsm[(size_t)L * kChunkFloats + fs * 32u + ln];
        }
    }
    return true;
}

// ---------------------------------------------------------------------------
// Phase: solve on one thread-block cluster, state in shared memory
// ---------------------------------------------------------------------------
// ContactSolver.solve with a barrier after every colour batch, as in
// phase_solve, with the state the sweeps pass from SM to SM held in the
// cluster's shared memory instead of L2: body i lives in CTA i % C (slot
// i / C) and is read and written by the other CTAs through distributed
// shared memory.  Each CTA prepares and solves its own manifolds with their
// velocity-sweep fields (CP_NVEL per point; tangent2 is recomputed from the
// normal and tangent1) in its shared memory: with the packing grouped by
// owner (owner_groups == C), the manifolds of each colour whose home body it
// holds, so that most manifold steps touch local bodies only; else the
// colour's manifolds dealt round-robin (position lo + k + C j to CTA k).
// Static bodies (up to kMaxStaticReplicas) are copied into every CTA.  The
// position sweeps read the fields that do not change during the solve from
// the packed rows.  Every operation and its order per body is that of
// phase_solve, so the results are bit-identical.
//
// Returns false, before any barrier and in every block alike, when the state
// does not fit the shared memory given (smem_bytes); the caller then runs
// phase_solve.
template <class T>
__device__ __forceinline__ T* cluster_map(T* p, uint32_t rank) {
    unsigned long long r;
    asm("mapa.u64 %0, %1, %2;" : "=l"(r) : "l"(p), "r"(rank));
    return reinterpret_cast<T*>(r);
}

// Another CTA's copy of a shared-memory object: through the cluster's
// distributed shared memory, or the object itself for a one-CTA group.
template <class G, class T>
__device__ __forceinline__ T* group_map(T* p, uint32_t rank) {
    if constexpr (G::kDistributed) return cluster_map(p, rank);
    else return p;
}

constexpr uint32_t kMaxStaticReplicas = 32;

struct ClusterSolveSmem {
    DBody* body;     // bcap records
    DBody* rep;      // copies of the static bodies (nrep)
    uint32_t* stat;  // their body indices, ascending
    uint4* man;      // per local slot: body a, body b, points, flags
    float2* fr;      // per local slot: friction, restitution
    float* row;      // pcap x CP_NVEL floats, point-major, the slots' points one after another
    uint32_t* pos;   // per local slot: packed position
    uint32_t* po;    // per local slot: its first point in row
    uint32_t* base;  // per colour: first local slot of this CTA; [ncol]: its slot count
    uint32_t bcap, scap, pcap, nrep;
};
// manifold flags; a body read from a static copy has its copy's index at
// bits 8-15 (a) or 16-23 (b)
enum : uint32_t { CM_WA = 1u, CM_WB = 2u, CM_STATIC = 4u, CM_BAD = 8u, CM_RA = 16u, CM_RB = 32u };

// Bytes of the layout for bcap bodies, nrep static copies, scap manifold
// slots and pcap points.
__device__ __forceinline__ size_t cluster_smem_bytes(uint32_t bcap, uint32_t nrep, uint32_t scap, uint32_t pcap,
                                                     uint32_t ncol) {
    return (size_t)(bcap + nrep) * sizeof(DBody) +
           (size_t)scap * (sizeof(uint4) + sizeof(float2) + 2u * sizeof(uint32_t)) +
           (size_t)pcap * CP_NVEL * sizeof(float) + (size_t)(ncol + 1u) * sizeof(uint32_t) +
           (size_t)kMaxStaticReplicas * sizeof(uint32_t);
}

template <class G>
__device__ bool phase_solve_cluster(G& g, WorldDev& w, uint32_t M, uint32_t ncol, unsigned char* smem,
                                    uint32_t smem_bytes) {
    const StepCfg& cf = w.cfg;
    const uint32_t C = g.nblocks(), k = g.block(), t = threadIdx.x, T = blockDim.x;
    const uint32_t N = w.n_bodies;
    if (ncol > 256u || M > w.pair_cap) return false;
    // by owner when the packing is grouped so and the fullest CTA's share
    // fits; else round-robin over the same positions (any order inside a
    // colour will do), which balances the CTAs exactly
    bool by_owner = C > 1u && w.cfg.owner_groups == C && C <= kMaxOwnerGroups;
    // this CTA's manifolds of colour c: positions [first(c), first(c) + count(c))
    // by owner, else every C-th from lo + k
    auto count_of = [&](uint32_t c, uint32_t cta) -> uint32_t {
        if (by_owner) return w.ocnt[c * C + cta + 1u] - w.ocnt[c * C + cta];
        const uint32_t n = w.colour_cnt[c + 1u] - w.colour_cnt[c];
        return n > cta ? (n - 1u - cta) / C + 1u : 0u;
    };
    // every CTA's slots and points under both dealings, tallied by every
    // block at once from the packing's counts (one or two loads a thread,
    // then shared atomics; the same values, so the same verdicts, in every
    // block): [0] slots by owner, [1] slots round-robin, [2] points by owner,
    // [3] points round-robin
    __shared__ uint32_t s_tally[4][kMaxOwnerGroups];
    __shared__ int s_bad;
    if (C > kMaxOwnerGroups) return false;
    for (uint32_t x = t; x < 4u * kMaxOwnerGroups; x += T) (&s_tally[0][0])[x] = 0u;
    if (t == 0) s_bad = 0;
    __syncthreads();
    const bool owner_ok = by_owner;
    for (uint32_t x = t; x < ncol * C; x += T) {
        const uint32_t c = x / C, cta = x - c * C;
        const uint32_t lo = w.colour_cnt[c], hi = w.colour_cnt[c + 1u];
        if (cta == 0u && (hi < lo || hi > M)) s_bad = 1;
        const uint32_t n = hi - lo;
        const uint32_t rr = n > cta && hi >= lo ? (n - 1u - cta) / C + 1u : 0u;
        if (rr) atomicAdd(&s_tally[1][cta], rr);
        if (owner_ok) {
            const uint32_t o = w.ocnt[c * C + cta + 1u] - w.ocnt[c * C + cta];
            if (o) atomicAdd(&s_tally[0][cta], o);
        }
    }
    const bool tallied = C > 1u && w.cfg.owner_groups == C && C <= kMaxOwnerGroups;
    if (tallied && t < C) {
        s_tally[2][t] = w.ocnt[kOwnerPoints + t];
        s_tally[3][t] = w.ocnt[kOwnerPoints + kMaxOwnerGroups + t];
    }
    __syncthreads();
    if (s_bad) return false;
    // the most slots any CTA holds (the same verdict in every block)
    uint32_t need = 0;
    ClusterSolveSmem sm;
    sm.bcap = (N + C - 1u) / C;
    sm.nrep = w.n_static <= kMaxStaticReplicas ? w.n_static : 0u;
    // point rows that do not fit in shared memory may go to w.crow: a CTA's
    // last slots (the point offsets are a prefix in slot order, so once a
    // slot's rows spill every later slot's do), in that CTA's range of w.crow
    // (its offset: the points of the CTAs before it)
    uint32_t needp = 0, goff = 0, gtot = 0;
    for (int attempt = 0; attempt < 2; ++attempt) {
        need = 0;
        needp = 0;
        goff = 0;
        gtot = 0;
        for (uint32_t cta = 0; cta < C; ++cta) {
            const uint32_t n = s_tally[by_owner ? 0 : 1][cta];
            need = max(need, n);
            // points: the packing's tallies when it grouped for this cluster;
            // one CTA holds every point of the constraint set; else four a slot
            const uint32_t p = tallied ? s_tally[by_owner ? 2 : 3][cta]
                               : C == 1u ? *(volatile uint32_t*)&w.ctr[C_POINTS]
                                         : 4u * n;
            needp = max(needp, p);
            if (cta < k) goff += p;
            gtot += p;
        }
        const size_t fixed = cluster_smem_bytes(sm.bcap, sm.nrep, max(need, 1u), 0u, ncol);
        if (!by_owner ||
            (fixed <= smem_bytes &&
             (w.crow != nullptr || fixed + (size_t)max(needp, 1u) * CP_NVEL * sizeof(float) <= smem_bytes)))
            break;
        by_owner = false;
    }
    sm.scap = max(need, 1u);
    sm.pcap = max(needp, 1u);
    const size_t fixed = cluster_smem_bytes(sm.bcap, sm.nrep, sm.scap, 0u, ncol);
    if (fixed > smem_bytes) return false;
    // rows in shared memory (the rest spill)
    const uint32_t pcap_s = (uint32_t)min((size_t)sm.pcap, (smem_bytes - fixed) / (CP_NVEL * sizeof(float)));
    const bool spill = pcap_s < sm.pcap;
    if (spill && (w.crow == nullptr || (size_t)gtot > 4u * (size_t)w.pair_cap)) return false;
    if (t == 0 && k == 0) w.ctr[C_SWEEP] = spill ? SWEEP_SPILL : SWEEP_SHARED;
    {
        unsigned char* p = smem;
        sm.body = reinterpret_cast<DBody*>(p);
        p += (size_t)sm.bcap * sizeof(DBody);
        sm.rep = reinterpret_cast<DBody*>(p);
        p += (size_t)sm.nrep * sizeof(DBody);
        sm.man = reinterpret_cast<uint4*>(p);
        p += (size_t)sm.scap * sizeof(uint4);
        sm.fr = reinterpret_cast<float2*>(p);
        p += (size_t)sm.scap * sizeof(float2);
        sm.row = reinterpret_cast<float*>(p);
        p += (size_t)pcap_s * CP_NVEL * sizeof(float);
        sm.pos = reinterpret_cast<uint32_t*>(p);
        p += (size_t)sm.scap * sizeof(uint32_t);
        sm.po = reinterpret_cast<uint32_t*>(p);
        p += (size_t)sm.scap * sizeof(uint32_t);
        sm.base = reinterpret_cast<uint32_t*>(p);
        p += (size_t)(ncol + 1u) * sizeof(uint32_t);
        sm.stat = reinterpret_cast<uint32_t*>(p);
    }
    // this CTA's first slot per colour (ncol <= 256 <= T): a block scan
    {
        uint32_t total = 0;
        const uint32_t ex = block_excl_scan(t < ncol ? count_of(t, k) : 0u, &total);
        if (t < ncol) sm.base[t] = ex;
        if (t == 0) sm.base[ncol] = total;
    }
    // this CTA's bodies, and a copy of every static body
    for (uint32_t s = t; s < sm.bcap; s += T) {
        const uint32_t i = s * C + k;
        if (i < N) sm.body[s] = w.body[i];
    }
    for (uint32_t r = t; r < sm.nrep; r += T) {
        const uint32_t i = w.stat_idx[r];
        sm.stat[r] = i < N ? i : 0xFFFFFFFFu;
        if (i < N) sm.rep[r] = w.body[i];
    }
    __syncthreads();
    // the static copy holding body i, or -1
    auto rep_of = [&](uint32_t i) -> int32_t {
        uint32_t lo = 0, hi = sm.nrep;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (sm.stat[mid] < i) lo = mid + 1u;
            else hi = mid;
        }
        return lo < sm.nrep && sm.stat[lo] == i ? (int32_t)lo : -1;
    };
    // this CTA's manifolds: bodies, flags, friction, normals and impulses,
    // every slot at once (its colour by binary search over the slot bases)
    const uint32_t nsl0 = sm.base[ncol];
    for (uint32_t slot = t; slot < nsl0; slot += T) {
        {
            uint32_t lo = 0, hi = ncol;  // the last colour whose base is <= slot
            while (hi - lo > 1u) {
                const uint32_t mid = (lo + hi) >> 1;
                if (sm.base[mid] <= slot) lo = mid;
                else hi = mid;
            }
            const uint32_t c = lo, j = slot - sm.base[c];
            const uint32_t first = by_owner ? w.ocnt[c * C + k] : w.colour_cnt[c] + k, stride = by_owner ? 1u : C;
            const uint32_t pos = first + stride * j;
            uint4 mv = w.cm[pos];
            uint32_t fl = 0u;
            if (mv.x >= N || mv.y >= N || mv.z > 4u) {
                atomicOr(&w.ctr[C_ERROR], ERR_BOUNDS);
                mv = make_uint4(0u, 0u, 0u, CM_BAD);
            } else {
                const DBodyProp pa = w.prop[mv.x], pb = w.prop[mv.y];
                fl = (writable(pa) ? CM_WA : 0u) | (writable(pb) ? CM_WB : 0u) |
                     (pa.type == 0u && pb.type == 0u ? CM_STATIC : 0u);
                if (pa.type == 0u) {
                    const int32_t r = rep_of(mv.x);
                    if (r >= 0) fl |= CM_RA | ((uint32_t)r << 8);
                }
                if (pb.type == 0u) {
                    const int32_t r = rep_of(mv.y);
                    if (r >= 0) fl |= CM_RB | ((uint32_t)r << 16);
                }
                mv.w = fl;
            }
            sm.man[slot] = mv;
            sm.fr[slot] = w.cfr[pos];
            sm.pos[slot] = pos;
            sm.po[slot] = mv.z;
        }
    }
    __syncthreads();
    if (g.rank() == 0 && w.ts) w.ts[TS_SW_SLOTS] = global_ns();
    // each slot's first point: exclusive scan of the point counts in slot order
    const uint32_t nsl = sm.base[ncol];
    uint32_t carry = 0;
    for (uint32_t lo = 0; lo < nsl; lo += T) {
        const uint32_t slot = lo + t;
        const uint32_t v = slot < nsl ? sm.po[slot] : 0u;
        uint32_t tile = 0;
        const uint32_t ex = block_excl_scan(v, &tile);
        if (slot < nsl) sm.po[slot] = carry + ex;
        carry += tile;
    }
    const bool points_fit = carry <= sm.pcap;  // the same in every thread of this block
    if (!points_fit && t == 0) atomicOr(&w.ctr[C_ERROR], ERR_BOUNDS);
    __syncthreads();
    // a slot's first point row: in shared memory, or spilled to this CTA's
    // range of w.crow
    auto row_of = [&](uint32_t slot, uint32_t n) -> float* {
        const uint32_t po = sm.po[slot];
        return po + n <= pcap_s ? sm.row + (size_t)po * CP_NVEL : w.crow + ((size_t)goff + po) * CP_NVEL;
    };
    for (uint32_t slot = t; slot < nsl; slot += T) {
        uint4 mv = sm.man[slot];
        if (!points_fit) {
            // never with the packing's own tallies; skip every manifold here
            // rather than write past the rows
            mv.w |= CM_BAD;
            mv.z = 0u;
            sm.man[slot] = mv;
            continue;
        }
        const CPV vg = cpv_global(w, sm.pos[slot]), vs{row_of(slot, mv.z), 1u, CP_NVEL};
        // every point's fields loaded before any is stored (the stores would
        // otherwise hold each next point's loads back)
        F3 nn[4];
        float ni[4], t0[4], t1[4];
#pragma unroll
        for (uint32_t i = 0; i < 4u; ++i) {
            if (i < mv.z) {
                nn[i] = ld3(vg, CP_NX, i);
                ni[i] = cpr(vg, CP_NI, i);
                t0[i] = cpr(vg, CP_TI0, i);
                t1[i] = cpr(vg, CP_TI1, i);
            }
        }
#pragma unroll
        for (uint32_t i = 0; i < 4u; ++i) {
            if (i < mv.z) {
                st3(vs, CP_NX, i, nn[i]);
                cpr(vs, CP_NI, i) = ni[i];
                cpr(vs, CP_TI0, i) = t0[i];
                cpr(vs, CP_TI1, i) = t1[i];
            }
        }
    }
    if (g.rank() == 0 && w.ts) w.ts[TS_SW_ROWS] = global_ns();
    g.sync();  // every block's bodies are in place (and every block has started)
    if (g.rank() == 0 && w.ts) w.ts[TS_SW_SETUP] = global_ns();
    const SolveFlags sf = solve_flags(cf);
    const float h = cf.dt / (float)cf.substeps;
    const Soft soft = soft_params(cf.hertz, cf.damping_ratio, h);
    const float hinv = h > kEpsilon ? 1.0f / h : 0.0f;
    const Soft hard{0.f, 1.f, 1.f};
    const F3 grav{cf.gravity[0], cf.gravity[1], cf.gravity[2]};
    const bool has = M > 0u;
    const uint32_t nslot = sm.base[ncol];
    // body i's home CTA and its slot there (shift and mask for the usual
    // power-of-two cluster)
    const uint32_t csh = (C & (C - 1u)) == 0u ? (uint32_t)(__ffs(C) - 1) : 32u;
    auto home = [&](uint32_t i) { return csh < 32u ? i & (C - 1u) : i % C; };
    auto home_slot = [&](uint32_t i) { return csh < 32u ? i >> csh : i / C; };
    // body a (or b) of a manifold: its static copy here, else its home CTA's record
    auto body_a = [&](const uint4& mv) {
        return (mv.w & CM_RA) ? sm.rep + ((mv.w >> 8) & 0xFFu) : group_map<G>(sm.body + home_slot(mv.x), home(mv.x));
    };
    auto body_b = [&](const uint4& mv) {
        return (mv.w & CM_RB) ? sm.rep + ((mv.w >> 16) & 0xFFu) : group_map<G>(sm.body + home_slot(mv.y), home(mv.y));
    };
    // one manifold of a velocity-type sweep: 0 warm start, 1 velocity, 2 relax
    auto vel_item = [&](uint32_t slot, uint32_t kind) {
        const uint4 mv = sm.man[slot];
        if (mv.w & CM_BAD) return;
        if (kind != 0u && mv.z == 0u) return;
        DBody* pa = body_a(mv);
        DBody* pb = body_b(mv);
        const DBody A = *pa, B = *pb;
        BV a = bv_of(A, (mv.w & CM_WA) != 0u), b = bv_of(B, (mv.w & CM_WB) != 0u);
        float* rows = row_of(slot, mv.z);
        if (kind == 0u)
            warm_points_rows(rows, mv.z, cf.warm_scale, a, b, sf.friction);
        else
            velocity_points_rows(sf.friction, rows, mv.z, sm.fr[slot].x, kind == 1u ? soft : hard, kind == 1u, a,
                                 b);
        if (a.wr) {
            pa->v = make_float4(a.v.x, a.v.y, a.v.z, 0.f);
            pa->w = make_float4(a.w.x, a.w.y, a.w.z, 0.f);
        }
        if (b.wr) {
            pb->v = make_float4(b.v.x, b.v.y, b.v.z, 0.f);
            pb->w = make_float4(b.w.x, b.w.y, b.w.z, 0.f);
        }
    };
    auto sweep = [&](uint32_t kind) {
        for (uint32_t c = 0; c < ncol; ++c) {
            const uint32_t b0 = sm.base[c], cnt = sm.base[c + 1u] - b0;
            for (uint32_t j = t; j < cnt; j += T) vel_item(b0 + j, kind);
            g.sync();
        }
    };
    for (uint32_t s = 0; s < cf.substeps; ++s) {
        // applyGravity (solver.zig:564-605)
        for (uint32_t q = t; q < sm.bcap; q += T) {
            const uint32_t i = q * C + k;
            if (i >= N) break;
            const DBodyProp& pr = w.prop[i];
            if (!(pr.type == 2u && pr.sleeping == 0u)) continue;
            DBody& b = sm.body[q];
            float4 v = b.v, av = b.w;
            body_gravity(v, av, pr, grav, h);
            b.v = v;
            b.w = av;
        }
        g.sync();
        if (has) {
            // prepareConstraints: one thread per (slot, point).  (One thread
            // per slot, its bodies read once and its points' inputs loaded
            // together, was slower: 0.960 against 0.939 ms on the pile.)
            for (uint32_t it = t; it < 4u * nslot; it += T) {
                const uint32_t slot = it >> 2, i = it & 3u;
                const uint4 mv = sm.man[slot];
                if (i >= mv.z || (mv.w & CM_BAD)) continue;
                const DBody A = *body_a(mv), B = *body_b(mv);
                const BV a = bv_of(A, (mv.w & CM_WA) != 0u), b = bv_of(B, (mv.w & CM_WB) != 0u);
                prepare_point_s<false>(sf, cpv_global(w, sm.pos[slot]),
                                       CPV{row_of(slot, mv.z), 1u, CP_NVEL},
                                       sm.fr[slot].y, i,
                                       soft, hinv, a, qof(A.q), b, qof(B.q));
            }
            g.sync();
            if (cf.warm_starting && s == 0u) sweep(0u);
            for (uint32_t vi = 0; vi < cf.vel_iters; ++vi) sweep(1u);
        }
        // integratePositions (solver.zig:841-845, 341-356)
        for (uint32_t q = t; q < sm.bcap; q += T) {
            const uint32_t i = q * C + k;
            if (i >= N) break;
            const DBodyProp& pr = w.prop[i];
            if (pr.type == 0u || pr.sleeping) continue;
            DBody b = sm.body[q];
            body_integrate(b, pr, h, cf.disable_rotation != 0u);
            sm.body[q] = b;
        }
        g.sync();
        if (has) sweep(2u);
        // test hook: every body's state after this substep
        if (cf.record_substeps && w.subrec) {
            for (uint32_t q = t; q < sm.bcap; q += T) {
                const uint32_t i = q * C + k;
                if (i >= N) break;
                const DBody b = sm.body[q];
                float* r = w.subrec + ((size_t)s * N + i) * 13u;
                r[0] = b.p.x; r[1] = b.p.y; r[2] = b.p.z;
                r[3] = b.q.x; r[4] = b.q.y; r[5] = b.q.z; r[6] = b.q.w;
                r[7] = b.v.x; r[8] = b.v.y; r[9] = b.v.z;
                r[10] = b.w.x; r[11] = b.w.y; r[12] = b.w.z;
            }
            if (g.rank() == 0) w.ctr[C_SUBREC] = s + 1u;
        }
    }
    if (g.rank() == 0 && w.ts) w.ts[TS_SW_SUBSTEPS] = global_ns();
    // the velocity sweeps are done: impulses and masses back to the packed
    // rows now (storeImpulses reads them), and in their rows each point's
    // position-sweep inputs, which do not change during the solve (the normal
    // stays where it is)
    const bool pos_rows = has && cf.pos_iters > 0u;
    if (pos_rows) {
        for (uint32_t slot = t; slot < nslot; slot += T) {
            const uint4 mv = sm.man[slot];
            const CPV vg = cpv_global(w, sm.pos[slot]);
            float* rows = row_of(slot, mv.z);
            // the packed inputs of every point loaded first, then the rows
            // rewritten (stores would otherwise hold the next loads back)
            F3 la[4], lb[4];
            float base[4];
#pragma unroll
            for (uint32_t i = 0; i < 4u; ++i) {
                if (i < mv.z) {
                    la[i] = ld3(vg, CP_LAX, i);
                    lb[i] = ld3(vg, CP_LBX, i);
                    base[i] = cpr(vg, CP_BASE, i);
                }
            }
#pragma unroll
            for (uint32_t i = 0; i < 4u; ++i) {
                if (i < mv.z) {
                    float* r = rows + (size_t)i * CP_NVEL;
                    cpr(vg, CP_NM, i) = r[CP_NM];
                    cpr(vg, CP_TM0, i) = r[CP_TM0];
                    cpr(vg, CP_TM1, i) = r[CP_TM1];
                    cpr(vg, CP_NI, i) = r[CP_NI];
                    cpr(vg, CP_TI0, i) = r[CP_TI0];
                    cpr(vg, CP_TI1, i) = r[CP_TI1];
                    r[CP_PX] = la[i].x; r[CP_PX + 1u] = la[i].y; r[CP_PX + 2u] = la[i].z;
                    r[CP_RAX] = lb[i].x; r[CP_RAX + 1u] = lb[i].y; r[CP_RAX + 2u] = lb[i].z;
                    r[CP_RBX] = base[i];
                }
            }
        }
        __syncthreads();  // the rows of this CTA are its own
    }
    if (has) {
        for (uint32_t it = 0; it < cf.pos_iters; ++it) {
            float mn = 0.0f, mx = -__int_as_float(0x7f800000);
            for (uint32_t c = 0; c < ncol; ++c) {
                const uint32_t b0 = sm.base[c], cnt = sm.base[c + 1u] - b0;
                for (uint32_t j = t; j < cnt; j += T) {
                    const uint32_t slot = b0 + j;
                    const uint4 mv = sm.man[slot];
                    if (mv.w & (CM_BAD | CM_STATIC)) continue;
                    DBody* pa = body_a(mv);
                    DBody* pb = body_b(mv);
                    const DBody A = *pa, B = *pb;
                    PB a = pb_of(A.p, A.q, A.i0, A.i1, A.i2, (mv.w & CM_WA) != 0u);
                    PB b = pb_of(B.p, B.q, B.i0, B.i1, B.i2, (mv.w & CM_WB) != 0u);
                    position_points_rows(sf, row_of(slot, mv.z), mv.z, a, b, &mn, &mx);
                    if (a.wr) {
                        pa->p = make_float4(a.x.x, a.x.y, a.x.z, a.im);
                        pa->q = f4of(a.q);
                    }
                    if (b.wr) {
                        pb->p = make_float4(b.x.x, b.x.y, b.x.z, b.im);
                        pb->q = f4of(b.q);
                    }
                }
                g.sync();
            }
            bool brk = false;
            pos_sweep_end(g, w, it, mn, mx, &brk);
            if (brk) break;
        }
    }
    g.sync();
    if (g.rank() == 0 && w.ts) w.ts[TS_SW_POSITION] = global_ns();
    // bodies back to the world, impulses and masses back to the packed rows
    // (storeImpulses reads them)
    for (uint32_t q = t; q < sm.bcap; q += T) {
        const uint32_t i = q * C + k;
        if (i >= N) break;
        if (w.prop[i].type != 0u) w.body[i] = sm.body[q];
    }
    for (uint32_t slot = pos_rows ? nslot : t; slot < nslot; slot += T) {  // done above when pos_rows
        const uint4 mv = sm.man[slot];
        const CPV vg = cpv_global(w, sm.pos[slot]), vs{row_of(slot, mv.z), 1u, CP_NVEL};
        for (uint32_t i = 0; i < mv.z; ++i) {
            cpr(vg, CP_NM, i) = cpr(vs, CP_NM, i);
            cpr(vg, CP_TM0, i) = cpr(vs, CP_TM0, i);
            cpr(vg, CP_TM1, i) = cpr(vs, CP_TM1, i);
            cpr(vg, CP_NI, i) = cpr(vs, CP_NI, i);
            cpr(vg, CP_TI0, i) = cpr(vs, CP_TI0, i);
            cpr(vg, CP_TI1, i) = cpr(vs, CP_TI1, i);
        }
    }
    return true;
}

// ---------------------------------------------------------------------------
// Phase: store (writeBack, storeImpulses, updateSleepStates)
// ---------------------------------------------------------------------------
template <class G>
__device__ bool phase_store(G& g, WorldDev& w, uint32_t cur, uint32_t M, bool solved) {
    const StepCfg& cf = w.cfg;
    for (uint32_t i = g.rank(); i < w.n_bodies; i += g.size()) {
        DBodyProp& pr = w.prop[i];
        if (pr.type == 0u) continue;
        DBody& b = w.body[i];
        F3 x = f3of(b.p), v = f3of(b.v), av = f3of(b.w);
        Qt q = qof(b.q);
        // BodyState.writeBack (solver.zig:246-296); skipped with the rest of
        // ContactSolver.solve when dt <= 0 (solver.zig:495)
        const bool qf = isfinite(q.x) && isfinite(q.y) && isfinite(q.z) && isfinite(q.w);
        if (solved && (!finite3(x) || !qf)) {
            const F3 x0 = f3of(w.p0[i]);
            x = finite3(x0) ? x0 : F3{0.f, 2.f, 0.f};
            q = Qt{0.f, 0.f, 0.f, 1.f};
            v = F3{0.f, 0.f, 0.f};
            av = F3{0.f, 0.f, 0.f};
        }
        if (solved) {
            if (!finite3(v)) v = F3{0.f, 0.f, 0.f};
            if (!finite3(av)) av = F3{0.f, 0.f, 0.f};
            const float ls2 = lensq3(v), as2 = lensq3(av);
            if (ls2 > 50.0f * 50.0f) v = v * (50.0f / sqrtf(ls2));
            if (as2 > 30.0f * 30.0f) av = av * (30.0f / sqrtf(as2));
            if (ls2 < 0.002f) v = F3{0.f, 0.f, 0.f};
            if (as2 < 0.002f) av = F3{0.f, 0.f, 0.f};
            q = qnormalize(q);
        }
        // VoxelBody.updateSleepState (body.zig:415-427) for awake dynamic bodies
        if (cf.sleeping_on && pr.type == 2u && !pr.sleeping) {
            if (len3(v) < 0.1f && len3(av) < 0.1f) {
                pr.sleep_timer += cf.dt;
                if (pr.sleep_timer >= 0.5f) {
                    pr.sleeping = 1u;
                    v = F3{0.f, 0.f, 0.f};
                    av = F3{0.f, 0.f, 0.f};
                }
            } else {
                pr.sleep_timer = 0.0f;
            }
        }
        b.p = make_float4(x.x, x.y, x.z, b.p.w);
        b.q = f4of(q);
        b.v = make_float4(v.x, v.y, v.z, 0.f);
        b.w = make_float4(av.x, av.y, av.z, 0.f);
    }
    // storeImpulses (solver.zig:933-958)
    if (solved && cf.warm_store_on) {
        for (uint32_t pos = g.rank(); pos < M; pos += g.size()) {
            const uint4 cmv = w.cm[pos];
            ManifoldRec& m = w.man[cur][cmv.w];
            const uint32_t n = cmv.z < m.n ? cmv.z : m.n;
            for (uint32_t i = 0; i < n; ++i) {
                m.c[i].normal_impulse = w.cp[cpi(w, CP_NI, i, pos)];
                m.c[i].tangent_impulse[0] = w.cp[cpi(w, CP_TI0, i, pos)];
                m.c[i].tangent_impulse[1] = w.cp[cpi(w, CP_TI1, i, pos)];
                m.c[i].normal_mass = w.cp[cpi(w, CP_NM, i, pos)];
                m.c[i].tangent_mass[0] = w.cp[cpi(w, CP_TM0, i, pos)];
                m.c[i].tangent_mass[1] = w.cp[cpi(w, CP_TM1, i, pos)];
            }
        }
    }
    return true;
}

// ---------------------------------------------------------------------------
// One whole step (VoxelPhysicsSystem.step with the pairs given)
// ---------------------------------------------------------------------------
template <class G>
__device__ __forceinline__ void stamp(G& g, WorldDev& w, uint32_t slot) {
    if (g.rank() == 0 && w.ts) w.ts[slot] = global_ns();
}

// The narrow part of one step: counters, begin (all-sleeping skip, world
// inverse inertia), the pair list, the narrow phase.  Returns true, and
// leaves C_SOLVE_GO set, when the solve part of the step is to run.
template <class G>
__device__ bool world_step_narrow(G& g, WorldDev& w, const ColliderSet& cs, WarpManifold* warp_sm,
                                  const CacheSmem& csm) {
    const uint32_t ph = w.cfg.phases;
    const uint32_t f0 = *(volatile uint32_t*)&w.frame[0];
    stamp(g, w, TS_START);
    if (w.n_bodies == 0u) return false;  // an empty batch slot
    // per-step counters (the sticky error word excepted)
    if (g.rank() < C_ERROR) w.ctr[g.rank()] = 0u;
    if (!g.sync()) return false;
    bool skipped = false;
    if (!phase_begin(g, w, (ph & PH_SKIP_TEST) != 0u, &skipped)) return false;
    stamp(g, w, TS_BEGIN);
    if (skipped) return false;
    if ((ph & PH_NARROW) && w.cfg.device_pairs) {
        bool overflow = false;
        if (!phase_broadphase(g, w, cs, &overflow, reinterpret_cast<unsigned char*>(warp_sm))) return false;
        stamp(g, w, TS_BROAD);
        if (overflow) {
            if (g.rank() == 0) atomicOr(&w.ctr[C_ERROR], ERR_CAP);
            return false;
        }
    } else {
        w.n_pairs = *w.n_pairs_dev;
        if ((ph & PH_NARROW) && w.n_pairs > w.pair_cap) {
            // the pair list did not fit: leave every state untouched, the
            // host grows the buffers and runs the step again
            if (g.rank() == 0) atomicOr(&w.ctr[C_ERROR], ERR_CAP);
            return false;
        }
    }
    // ContactManager.beginFrame (narrow_phase.zig:1003-1008): the previous
    // "current" manifolds become "previous"
    if (ph & PH_NARROW) {
        const uint32_t cur = (f0 + 1u) & 1u, prev = cur ^ 1u;
        if (g.rank() == 0) {
            w.frame[0] = f0 + 1u;
            w.frame[1] = w.n_pairs;
        }
        if (!phase_pairs(g, w, cs, cur)) return false;
        stamp(g, w, TS_PAIRS);
        stamp(g, w, TS_CACHE);
        if (!phase_probe(g, w, cs, cur, warp_sm, csm)) return false;
        stamp(g, w, TS_PROBE);
        if (!phase_finalize(g, w, cur, prev)) return false;
        stamp(g, w, TS_FINALIZE);
    }
    if (g.rank() == 0) w.ctr[C_SOLVE_GO] = 1u;
    return g.sync();
}

// How much of the solve part one launch runs.
enum : uint32_t {
    SOLVE_ALL = 0,          // constraints, colouring, sweeps, store
    SOLVE_CONSTRAINTS = 1,  // constraints and colouring; world_step_sweeps runs the rest
};

// The solve part of one step: constraints, colouring, ContactSolver.solve,
// store and sleep.  check_go: read the narrow part's verdict from C_SOLVE_GO
// (the parts run as two kernels).  part SOLVE_CONSTRAINTS stops after the
// colouring and leaves M, ncol and C_SOLVE_GO = 2 for world_step_sweeps.
template <class G>
__device__ void world_step_solve(G& g, WorldDev& w, float* fsm, bool check_go, uint32_t part = SOLVE_ALL) {
    const uint32_t ph = w.cfg.phases;
    if (!(ph & PH_SOLVE) || w.n_bodies == 0u) return;
    if (check_go && *(volatile uint32_t*)&w.ctr[C_SOLVE_GO] == 0u) return;
    w.n_pairs = *(volatile uint32_t*)w.n_pairs_dev;
    const uint32_t cur = *(volatile uint32_t*)&w.frame[0] & 1u;  // the latest manifolds
    // The solver's work per colour batch is a few hundred manifolds: run it
    // on k blocks (one per solver_div manifolds, at least 2) with a cheaper
    // barrier.
    const uint32_t nman = (ph & PH_NARROW) ? *(volatile uint32_t*)&w.ctr[C_MANIFOLDS] : w.n_pairs;
    uint32_t want = max(2u, (nman + w.cfg.solver_div - 1u) / w.cfg.solver_div);
    // event-ordered sweeps: enough blocks to hold every chunk (at most
    // nman / 32 + one partial chunk per colour) in shared memory
    if (G::kEventSweeps && w.cfg.solver_flow && w.cfg.flow_smem_chunks)
        want = max(want, (nman / 32u + 64u + w.cfg.flow_smem_chunks - 1u) / w.cfg.flow_smem_chunks);
    G s = g.subgroup(min(want, g.nblocks()));
    // The island pass only reads (manifolds, velocities before the solve) and
    // writes statistics, so while the constraint table is built the blocks
    // that phase leaves idle run it, when the sweeps follow in another kernel.
    bool islands_here = true;
    if constexpr (G::kEventSweeps) {
        if (part == SOLVE_CONSTRAINTS && w.cfg.islands_on && want + 2u <= g.nblocks()) {
            islands_here = false;
            if (!s.member()) {
                G r = g.tail(want);
                phase_islands(r, w, cur, w.isl_state + IS_N);
                return;
            }
        }
    }
    if (!s.member()) return;
    uint32_t M = 0, ncol = 0;
    if (!phase_constraints(s, w, cur, &M, &ncol, islands_here)) return;
    stamp(s, w, TS_CONSTRAINTS);
    if (part == SOLVE_CONSTRAINTS) {
        if (s.rank() == 0) {
            w.ctr[C_CONS_M] = M;
            w.ctr[C_CONS_NCOL] = ncol;
            __threadfence();
            w.ctr[C_SOLVE_GO] = 2u;
        }
        return;
    }
    const bool solved = w.cfg.dt > 0.0f && w.n_bodies > 0u;
    // event-ordered sweeps unless a kinematic body (moved every substep,
    // written by nobody) sits in a constraint
    if (solved) {
        bool ok;
        if constexpr (G::kEventSweeps) {
            const bool flow = w.cfg.solver_flow && !w.cfg.record_substeps && w.cfg.vel_iters > 0u &&
                              w.cfg.substeps > 0u &&
                              *(volatile uint32_t*)&w.ctr[C_KIN_CONTACT] == 0u &&
                              (*(volatile uint32_t*)&w.ctr[C_ERROR] & ERR_COLOURS) == 0u;
            ok = flow ? phase_solve_flow(s, w, fsm, M, ncol) : phase_solve(s, w, M, ncol);
        } else {
            // a one-CTA world: the sweeps keep their state in the block's
            // shared memory when it fits (the narrow part is done with it)
            ok = (w.cfg.block_smem && phase_solve_cluster(s, w, M, ncol, reinterpret_cast<unsigned char*>(fsm),
                                                          w.cfg.block_smem)) ||
                 phase_solve(s, w, M, ncol);
        }
        if (!ok) return;
    }
    if (!s.sync()) return;
    stamp(s, w, TS_SOLVE);
    if (!phase_store(s, w, cur, M, solved)) return;
    stamp(s, w, TS_END);
}

// The solve part on one thread-block cluster.  whole: all of it (constraints,
// colouring, sweeps, store and sleep) right after the narrow part; else the
// part after world_step_solve(..., SOLVE_CONSTRAINTS) on the grid.  The
// sweeps run by phase_solve_cluster (state in shared memory) or, when that
// does not fit, phase_solve.  Every block reads the go flag, M and ncol
// (written by the previous kernel, or by this one before a barrier) and
// passes the same barriers: their number follows from those values, the
// configuration, the colouring's round count and the position sweeps' early
// break, which every block reads from a slot that no block writes again
// before the next barrier.
__device__ __forceinline__ void world_step_sweeps(ClusterGroup& g, WorldDev& w, unsigned char* smem,
                                                  uint32_t smem_bytes, bool whole) {
    const uint32_t ph = w.cfg.phases;
    if (!(ph & PH_SOLVE) || w.n_bodies == 0u) return;
    if (*(volatile uint32_t*)&w.ctr[C_SOLVE_GO] != (whole ? 1u : 2u)) return;
    w.n_pairs = *(volatile uint32_t*)w.n_pairs_dev;
    const uint32_t cur = *(volatile uint32_t*)&w.frame[0] & 1u;
    uint32_t M, ncol;
    if (whole) {
        phase_constraints(g, w, cur, &M, &ncol);
        stamp(g, w, TS_CONSTRAINTS);
    } else {
        M = *(volatile uint32_t*)&w.ctr[C_CONS_M];
        ncol = *(volatile uint32_t*)&w.ctr[C_CONS_NCOL];
        // the position sweeps' min-separation slots at this group's offset
        if (g.rank() < 16u) w.scan[g.nblocks() + 4u + g.rank()] = 0u;
        g.sync();
    }
    const bool solved = w.cfg.dt > 0.0f;
    if (solved && !phase_solve_cluster(g, w, M, ncol, smem, smem_bytes)) {
        if (g.rank() == 0) w.ctr[C_SWEEP] = SWEEP_L2;
        phase_solve(g, w, M, ncol);
    }
    g.sync();
    stamp(g, w, TS_SOLVE);
    phase_store(g, w, cur, M, solved);
    stamp(g, w, TS_END);
}

// One whole step (VoxelPhysicsSystem.step with the pairs given) in one
// kernel: the narrow part, then the solve part.
template <class G>
__device__ void world_step(G& g, WorldDev& w, const ColliderSet& cs, WarpManifold* warp_sm, const CacheSmem& csm,
                           float* fsm) {
    if (world_step_narrow(g, w, cs, warp_sm, csm)) world_step_solve(g, w, fsm, false);
}

}  // namespace vxp
