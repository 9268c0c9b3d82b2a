// oracle_capi.cpp — C entry points over vxp_oracle.hpp for the Python tests
// and for bench.py's CPU-baseline leg.  TEST INFRASTRUCTURE ONLY.
//
// The structs are the ones the product's C ABI uses (include/vxp.h) so that a
// test can hand the same buffers to the oracle and to the CUDA library.
#include "vxp_oracle.hpp"

#include <atomic>
#include <cstdio>
#include <memory>
#include <thread>

#include "../include/vxp.h"

using namespace vxo;

namespace {

template <class R> Body<R> toBody(const vxp_body& s, const std::unordered_map<uint32_t, int32_t>& cmap) {
    Body<R> b;
    b.id = s.id;
    b.type = s.body_type;
    auto it = cmap.find(s.collider_id);
    b.collider = it == cmap.end() ? -1 : it->second;
    b.sleeping = s.is_sleeping != 0;
    b.pos = {(R)s.position[0], (R)s.position[1], (R)s.position[2]};
    b.rot = {(R)s.rotation[0], (R)s.rotation[1], (R)s.rotation[2], (R)s.rotation[3]};
    b.v = {(R)s.linear_velocity[0], (R)s.linear_velocity[1], (R)s.linear_velocity[2]};
    b.w = {(R)s.angular_velocity[0], (R)s.angular_velocity[1], (R)s.angular_velocity[2]};
    b.inv_mass = (R)s.inv_mass;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) b.inv_I_local.m[i][j] = (R)s.inv_inertia_local[i * 3 + j];
    b.friction = (R)s.friction;
    b.restitution = (R)s.restitution;
    b.lin_damp = (R)s.linear_damping;
    b.ang_damp = (R)s.angular_damping;
    b.sleep_timer = (R)s.sleep_timer;
    return b;
}
template <class R> void fromBody(const Body<R>& b, uint32_t collider_id, vxp_body* s) {
    s->id = b.id;
    s->body_type = b.type;
    s->collider_id = collider_id;
    s->is_sleeping = b.sleeping ? 1u : 0u;
    s->position[0] = (float)b.pos.x; s->position[1] = (float)b.pos.y; s->position[2] = (float)b.pos.z;
    s->rotation[0] = (float)b.rot.x; s->rotation[1] = (float)b.rot.y;
    s->rotation[2] = (float)b.rot.z; s->rotation[3] = (float)b.rot.w;
    s->linear_velocity[0] = (float)b.v.x; s->linear_velocity[1] = (float)b.v.y; s->linear_velocity[2] = (float)b.v.z;
    s->angular_velocity[0] = (float)b.w.x; s->angular_velocity[1] = (float)b.w.y; s->angular_velocity[2] = (float)b.w.z;
    s->inv_mass = (float)b.inv_mass;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) s->inv_inertia_local[i * 3 + j] = (float)b.inv_I_local.m[i][j];
    s->friction = (float)b.friction;
    s->restitution = (float)b.restitution;
    s->linear_damping = (float)b.lin_damp;
    s->angular_damping = (float)b.ang_damp;
    s->sleep_timer = (float)b.sleep_timer;
}

struct HandleBase {
    virtual ~HandleBase() = default;
};

template <class R> struct Handle : HandleBase {
    World<R> w;
    std::unordered_map<uint32_t, int32_t> cmap;   // collider id -> index
    std::vector<uint32_t> body_collider_id;        // per body, the public id
    Handle(const WorldConfig& wc, const SolverConfig<R>& sc) : w(wc, sc) {}
};

struct Any {
    int prec;
    std::unique_ptr<HandleBase> h;
};

WorldConfig toWorldCfg(const vxp_config* c) {
    WorldConfig w;
    for (int i = 0; i < 3; ++i) w.gravity[i] = c->gravity[i];
    w.fixed_timestep = c->fixed_timestep;
    w.enable_sleeping = c->enable_sleeping != 0;
    w.enable_warm_starting = c->enable_warm_starting != 0;
    w.use_brick_sat = c->use_brick_sat != 0;
    w.use_brick_pair_cache = c->use_brick_pair_cache != 0;
    w.cache_size = c->brick_pair_cache_size ? c->brick_pair_cache_size : 1024;
    w.reference_caps = c->reference_caps != 0;
    w.colouring = c->colouring;
    w.enable_islands = c->enable_islands != 0;
    return w;
}
template <class R> SolverConfig<R> toSolverCfg(const vxp_config* c) {
    SolverConfig<R> s;
    s.substeps = c->substeps;
    s.velocity_iterations = c->velocity_iterations;
    s.position_iterations = c->position_iterations;
    s.disable_rotation = c->disable_rotation != 0;
    s.hertz = (R)c->hertz;
    s.damping_ratio = (R)c->damping_ratio;
    s.position_correction_rate = (R)c->position_correction_rate;
    s.max_position_correction = (R)c->max_position_correction;
    s.slop = (R)c->slop;
    s.warm_starting = c->warm_starting != 0;
    s.warm_start_scale = (R)c->warm_start_scale;
    s.gravity = {(R)c->gravity[0], (R)c->gravity[1], (R)c->gravity[2]};
    s.enable_friction = c->enable_friction != 0;
    s.enable_restitution = c->enable_restitution != 0;
    return s;
}

template <class R> Handle<R>* H(void* p) { return static_cast<Handle<R>*>(static_cast<Any*>(p)->h.get()); }
int prec(void* p) { return static_cast<Any*>(p)->prec; }

#define DISPATCH(p, call)                    \
    do {                                     \
        if (prec(p) == 64) {                 \
            auto* h = H<double>(p);          \
            call;                            \
        } else {                             \
            auto* h = H<float>(p);           \
            call;                            \
        }                                    \
    } while (0)

template <class R> std::vector<std::pair<uint32_t, uint32_t>> toPairs(const vxp_pair* p, uint32_t n) {
    std::vector<std::pair<uint32_t, uint32_t>> v(n);
    for (uint32_t i = 0; i < n; ++i) v[i] = {p[i].body_a, p[i].body_b};
    return v;
}

template <class R> void manifoldOut(const Manifold<R>& m, vxp_manifold* o) {
    std::memset(o, 0, sizeof(*o));
    o->body_a_id = m.a;
    o->body_b_id = m.b;
    o->contact_count = m.n;
    o->friction = (float)m.friction;
    o->restitution = (float)m.restitution;
    for (uint32_t i = 0; i < m.n; ++i) {
        const Contact<R>& c = m.c[i];
        vxp_contact& k = o->contacts[i];
        k.point[0] = (float)c.point.x; k.point[1] = (float)c.point.y; k.point[2] = (float)c.point.z;
        k.normal[0] = (float)c.normal.x; k.normal[1] = (float)c.normal.y; k.normal[2] = (float)c.normal.z;
        k.penetration = (float)c.penetration;
        k.local_anchor_a[0] = (float)c.la.x; k.local_anchor_a[1] = (float)c.la.y; k.local_anchor_a[2] = (float)c.la.z;
        k.local_anchor_b[0] = (float)c.lb.x; k.local_anchor_b[1] = (float)c.lb.y; k.local_anchor_b[2] = (float)c.lb.z;
        k.normal_impulse = (float)c.normal_impulse;
        k.tangent_impulse[0] = (float)c.tangent_impulse[0];
        k.tangent_impulse[1] = (float)c.tangent_impulse[1];
        k.normal_mass = (float)c.normal_mass;
        k.tangent_mass[0] = (float)c.tangent_mass[0];
        k.tangent_mass[1] = (float)c.tangent_mass[1];
        k.feature_id = c.feature_id;
    }
}

template <class R>
int readCollider(Handle<R>& h, uint32_t collider_id, vxp_collider_info* info, vxp_brick* bricks, uint32_t cap,
                 uint32_t* n_out) {
    auto it = h.cmap.find(collider_id);
    if (it == h.cmap.end()) return VXP_ERR_ARG;
    const Collider<R>& c = h.w.colliders[(size_t)it->second];
    const uint32_t n = (uint32_t)c.bricks.size();
    if (info) {
        std::memset(info, 0, sizeof(*info));
        info->voxel_size = (float)c.voxel_size;
        const int32_t mn[3] = {c.min_bound.x, c.min_bound.y, c.min_bound.z};
        const int32_t mx[3] = {c.max_bound.x, c.max_bound.y, c.max_bound.z};
        const R amn[3] = {c.local_aabb.mn.x, c.local_aabb.mn.y, c.local_aabb.mn.z};
        const R amx[3] = {c.local_aabb.mx.x, c.local_aabb.mx.y, c.local_aabb.mx.z};
        for (int k = 0; k < 3; ++k) {
            info->min_bound[k] = mn[k];
            info->max_bound[k] = mx[k];
            info->aabb_min[k] = (float)amn[k];
            info->aabb_max[k] = (float)amx[k];
        }
        info->solid_count = c.solid_count;
        info->n_bricks = n;
    }
    if (n_out) *n_out = n;
    for (uint32_t b = 0; bricks && b < std::min(cap, n); ++b) {
        bricks[b].pos[0] = c.bricks[b].pos.x;
        bricks[b].pos[1] = c.bricks[b].pos.y;
        bricks[b].pos[2] = c.bricks[b].pos.z;
        std::memcpy(bricks[b].voxels, c.bricks[b].vox, 512);
    }
    return VXP_OK;
}

Obb<float> obbIn(const float* a) {
    return {{a[0], a[1], a[2]}, {a[3], a[4], a[5]}, {a[6], a[7], a[8], a[9]}};
}

}  // namespace

extern "C" {

void* vxo_world_create(const vxp_config* cfg, int precision) {
    Any* a = new Any;
    a->prec = precision == 64 ? 64 : 32;
    if (a->prec == 64) a->h.reset(new Handle<double>(toWorldCfg(cfg), toSolverCfg<double>(cfg)));
    else a->h.reset(new Handle<float>(toWorldCfg(cfg), toSolverCfg<float>(cfg)));
    return a;
}
void vxo_world_destroy(void* p) { delete static_cast<Any*>(p); }

int vxo_collider_add(void* p, uint32_t collider_id, float vs, const vxp_brick* bricks, uint32_t n) {
    std::vector<IV3> pos(n);
    std::vector<uint8_t> vox((size_t)n * 512);
    for (uint32_t i = 0; i < n; ++i) {
        pos[i] = {bricks[i].pos[0], bricks[i].pos[1], bricks[i].pos[2]};
        std::memcpy(&vox[(size_t)i * 512], bricks[i].voxels, 512);
    }
    int rc = 0;
    DISPATCH(p, {
        using R = std::remove_reference_t<decltype(h->w.colliders[0].voxel_size)>;
        Collider<R> c;
        if (!c.build((R)vs, pos.data(), vox.data(), n)) {
            rc = VXP_ERR_ARG;
        } else {
            auto it = h->cmap.find(collider_id);
            if (it != h->cmap.end()) h->w.colliders[(size_t)it->second] = c;
            else {
                h->cmap[collider_id] = (int32_t)h->w.colliders.size();
                h->w.colliders.push_back(c);
            }
        }
    });
    return rc;
}

int vxo_collider_edit(void* p, uint32_t collider_id, const int32_t* coords, const uint8_t* values, uint32_t n,
                      int mode) {
    if (mode != 0 && mode != 1) return VXP_ERR_ARG;
    int rc = 0;
    DISPATCH(p, {
        auto it = h->cmap.find(collider_id);
        if (it == h->cmap.end()) rc = VXP_ERR_ARG;
        else h->w.colliders[(size_t)it->second].edit(coords, values, n, mode);
    });
    return rc;
}

int vxo_collider_read(void* p, uint32_t collider_id, vxp_collider_info* info, vxp_brick* bricks, uint32_t cap,
                      uint32_t* n_out) {
    int rc = 0;
    DISPATCH(p, rc = readCollider(*h, collider_id, info, bricks, cap, n_out));
    return rc;
}

uint32_t vxo_invalidate_cache_for_body(void* p, uint32_t body_id) {
    uint32_t n = 0;
    DISPATCH(p, {
        const uint64_t before = h->w.cache.invalidations;
        h->w.cache.invalidateBody(body_id);
        n = (uint32_t)(h->w.cache.invalidations - before);
    });
    return n;
}

int vxo_bodies_set(void* p, const vxp_body* b, uint32_t n) {
    DISPATCH(p, {
        using R = std::remove_reference_t<decltype(h->w.bodies[0].inv_mass)>;
        h->w.bodies.resize(n);
        h->body_collider_id.resize(n);
        for (uint32_t i = 0; i < n; ++i) {
            h->w.bodies[i] = toBody<R>(b[i], h->cmap);
            h->body_collider_id[i] = b[i].collider_id;
        }
        h->w.reindex();
        h->w.islands.markDirty();  // the bodies were replaced: rebuild at the next solve
    });
    return 0;
}

int vxo_bodies_get(void* p, vxp_body* b, uint32_t n) {
    int rc = 0;
    DISPATCH(p, {
        if (n != h->w.bodies.size()) rc = VXP_ERR_ARG;
        else
            for (uint32_t i = 0; i < n; ++i) fromBody(h->w.bodies[i], h->body_collider_id[i], &b[i]);
    });
    return rc;
}

int vxo_step(void* p, float dt, const vxp_pair* pairs, uint32_t n) {
    DISPATCH(p, {
        using R = std::remove_reference_t<decltype(h->w.bodies[0].inv_mass)>;
        h->w.step((R)dt, toPairs<R>(pairs, n));
    });
    return 0;
}

// narrowPhase() alone (no sleep skip test), then vxo_solve for solve()+sleep.
int vxo_narrow_phase(void* p, const vxp_pair* pairs, uint32_t n) {
    DISPATCH(p, {
        using R = std::remove_reference_t<decltype(h->w.bodies[0].inv_mass)>;
        h->w.stats = Stats{};
        h->w.stats.pairs_in = n;
        h->w.narrowPhase(toPairs<R>(pairs, n));
    });
    return 0;
}
int vxo_solve(void* p, float dt) {
    DISPATCH(p, {
        using R = std::remove_reference_t<decltype(h->w.bodies[0].inv_mass)>;
        h->w.solve((R)dt);
        if (h->w.wcfg.enable_sleeping)
            for (auto& b : h->w.bodies)
                if (b.type == B_DYNAMIC && !b.sleeping) b.updateSleepState((R)dt);
    });
    return 0;
}

int vxo_manifolds_get(void* p, vxp_manifold* out, uint32_t cap, uint32_t* n_out) {
    DISPATCH(p, {
        const uint32_t n = (uint32_t)std::min<size_t>(cap, h->w.cm.cur.size());
        for (uint32_t i = 0; i < n; ++i) manifoldOut(h->w.cm.cur[i], &out[i]);
        *n_out = (uint32_t)h->w.cm.cur.size();
    });
    return 0;
}

int vxo_stats_get(void* p, vxp_stats* s) {
    DISPATCH(p, {
        const Stats& t = h->w.stats;
        s->pairs_in = t.pairs_in;
        s->pairs_tested = t.pairs_tested;
        s->pairs_colliding = t.pairs_colliding;
        s->voxels_checked = t.voxels_checked;
        s->contacts_generated = t.contacts_generated;
        s->pairs_skipped_sleeping = t.pairs_skipped_sleeping;
        s->manifolds_preserved = t.manifolds_preserved;
        s->cache_hits = t.cache_hits;
        s->cache_misses = t.cache_misses;
        s->cache_evictions = t.cache_evictions;
        s->manifolds = t.manifolds;
        s->constraints = t.constraints;
        s->contact_points = t.contact_points;
        s->colours = t.colours;
        s->position_iterations_run = t.position_iterations_run;
        s->step_skipped = t.step_skipped;
        s->max_penetration = t.max_penetration;
        s->candidates = t.candidates;
        s->island_count = t.island_count;
        s->active_islands = t.active_islands;
        s->sleeping_islands = t.sleeping_islands;
        s->largest_island_size = t.largest_island_size;
    });
    return 0;
}

int vxo_colours_get(void* p, uint32_t* out, uint32_t cap, uint32_t* n_out) {
    int overflow = 0;
    DISPATCH(p, {
        const uint32_t n = (uint32_t)std::min<size_t>(cap, h->w.last_colours.size());
        for (uint32_t i = 0; i < n; ++i) out[i] = h->w.last_colours[i];
        *n_out = (uint32_t)h->w.last_colours.size();
        overflow = h->w.colouring_overflow ? 1 : 0;
    });
    return overflow;
}

// Per-substep body states of the last solve (test hook): 13 floats per body
// per substep (position, rotation, linear and angular velocity).
int vxo_set_substep_record(void* p, int on) {
    DISPATCH(p, { h->w.solver.record_substeps = on != 0; });
    return 0;
}
int vxo_substeps_get(void* p, float* out, uint32_t cap_floats, uint32_t* n_substeps) {
    DISPATCH(p, {
        const auto& g = h->w.solver.substep_log;
        const size_t n = std::min<size_t>(cap_floats, g.size());
        for (size_t i = 0; i < n; ++i) out[i] = g[i];
        *n_substeps = h->w.solver.substeps_logged;
    });
    return 0;
}

int vxo_set_candidate_dump(void* p, int on) {
    DISPATCH(p, { h->w.dump = on != 0; });
    return 0;
}
int vxo_candidates_get(void* p, vxp_candidate* out, uint32_t cap, uint32_t* n_out) {
    DISPATCH(p, {
        const auto& c = h->w.candidates;
        const uint32_t n = (uint32_t)std::min<size_t>(cap, c.size());
        for (uint32_t i = 0; i < n; ++i) {
            out[i].pair_index = c[i].pair_index;
            out[i].a[0] = c[i].a.x; out[i].a[1] = c[i].a.y; out[i].a[2] = c[i].a.z;
            out[i].b[0] = c[i].b.x; out[i].b[1] = c[i].b.y; out[i].b[2] = c[i].b.z;
            out[i].passed = c[i].passed;
            out[i].dist_sq = c[i].dist_sq;
        }
        *n_out = (uint32_t)c.size();
    });
    return 0;
}

// IslandManager.buildIslands / buildIslandsWithBodyTypes over n manifolds
// given as (body_a, body_b) pairs (the reference's own island tests,
// islands.zig:785-816 and 857-888).  types: BodyType per body id (ntypes of
// them), or null for buildIslands.  island_of[id] (n_ids entries): the
// island index of body id, -1 for a body in no island.
int vxo_islands_kat(const vxp_pair* ms, uint32_t n, uint32_t body_count, const uint32_t* types, uint32_t ntypes,
                    int32_t* island_of, uint32_t n_ids, uint32_t* total_islands, uint32_t* largest) {
    IslandManager<float> m(body_count);
    std::vector<Manifold<float>> v(n);
    for (uint32_t i = 0; i < n; ++i) {
        v[i].a = ms[i].body_a;
        v[i].b = ms[i].body_b;
    }
    std::vector<uint32_t> t;
    if (types) t.assign(types, types + ntypes);
    m.build(v, body_count, t);
    for (uint32_t id = 0; id < n_ids; ++id) {
        auto it = m.body_to_island.find(id);
        island_of[id] = it == m.body_to_island.end() ? -1 : (int32_t)it->second;
    }
    *total_islands = (uint32_t)m.total_islands;
    *largest = (uint32_t)m.largest_island_size;
    return 0;
}

// VoxelBody.getWorldAABB (body.zig:430-435) of every body, 3 floats each.
int vxo_world_aabbs(void* p, float* mn, float* mx, uint32_t cap) {
    int rc = 0;
    DISPATCH(p, {
        const auto& bodies = h->w.bodies;
        if (bodies.size() > cap) {
            rc = VXP_ERR_CAP;
        } else {
            for (size_t i = 0; i < bodies.size(); ++i) {
                const auto& b = bodies[i];
                using R = std::remove_reference_t<decltype(b.inv_mass)>;
                Aabb<R> bx;  // a body without a collider: its position (no comma: this is a macro argument)
                bx.mn = b.pos;
                bx.mx = b.pos;
                if (b.collider >= 0) bx = aabbTransform(h->w.colliders[(size_t)b.collider].local_aabb, b.xf());
                mn[3 * i] = (float)bx.mn.x; mn[3 * i + 1] = (float)bx.mn.y; mn[3 * i + 2] = (float)bx.mn.z;
                mx[3 * i] = (float)bx.mx.x; mx[3 * i + 1] = (float)bx.mx.y; mx[3 * i + 2] = (float)bx.mx.z;
            }
        }
    });
    return rc;
}

int vxo_pairs_find(void* p, float margin, vxp_pair* out, uint32_t cap, uint32_t* n_out) {
    int rc = 0;
    DISPATCH(p, {
        using R = std::remove_reference_t<decltype(h->w.bodies[0].inv_mass)>;
        auto v = h->w.findPairs((R)margin);
        *n_out = (uint32_t)v.size();
        if (v.size() > cap) rc = VXP_ERR_CAP;
        for (uint32_t i = 0; i < std::min<size_t>(cap, v.size()); ++i) {
            out[i].body_a = v[i].first;
            out[i].body_b = v[i].second;
        }
    });
    return rc;
}

// Multi-threaded narrow phase with the reference's partitioning: T contiguous
// ranges of ceil(P/T) pairs, each processed by one thread into its own buffer,
// buffers merged in thread order (narrow_phase.zig:1538-1632).  As in
// ParallelNarrowPhaseContext, the brick-pair cache is read (hits replay) but
// never written (narrow_phase.zig:1231-1270).  f32 worlds only.  Returns the
// number of contacts generated.
static int narrow_threaded(World<float>& w, const vxp_pair* pairs, uint32_t n, int threads) {
    w.cm.beginFrame();
    w.cache.beginFrame();
    std::vector<uint32_t> filt;
    for (uint32_t i = 0; i < n; ++i) {
        Body<float>* a = w.find(pairs[i].body_a);
        Body<float>* b = w.find(pairs[i].body_b);
        const bool as = a ? a->sleeping : false, bs = b ? b->sleeping : false;
        if (as && bs) {
            const uint64_t key = pairKey(pairs[i].body_a, pairs[i].body_b);
            if (const Manifold<float>* pm = w.cm.prevGet(key)) w.cm.put(key, *pm);
            continue;
        }
        if (w.wcfg.reference_caps && filt.size() >= 512) continue;
        if (a && b) filt.push_back(i);
    }
    const int T = std::max(1, std::min(threads, 256));
    const size_t per = (filt.size() + (size_t)T - 1) / (size_t)T;
    std::vector<std::vector<Manifold<float>>> out((size_t)T);
    std::vector<std::thread> th;
    std::atomic<uint64_t> hits{0}, misses{0};
    for (int t = 0; t < T; ++t) {
        const size_t s0 = (size_t)t * per, e = std::min(filt.size(), s0 + per);
        if (s0 >= e) break;
        th.emplace_back([&, t, s0, e]() {
            for (size_t k = s0; k < e; ++k) {
                const Body<float>& a = *w.find(pairs[filt[k]].body_a);
                const Body<float>& b = *w.find(pairs[filt[k]].body_b);
                if (a.collider < 0 || b.collider < 0) continue;
                const Collider<float>& ca = w.colliders[(size_t)a.collider];
                const Collider<float>& cb = w.colliders[(size_t)b.collider];
                const Xf<float> ta = a.xf(), tb = b.xf();
                if (w.wcfg.use_brick_sat &&
                    satEarlyOut(obbFromAabb(ca.local_aabb, ta), obbFromAabb(cb.local_aabb, tb)))
                    continue;
                const bool use_cache = w.wcfg.use_brick_pair_cache &&
                                       (a.type == B_STATIC || b.type == B_STATIC || a.sleeping || b.sleeping);
                if (use_cache) {
                    // read-only lookup without touching LRU state (the
                    // reference mutates last_used_frame from several threads)
                    const V3<float> rp = sub(tb.p, ta.p);
                    const Q<float> rr = qmul(qconj(ta.q), tb.q);
                    const CacheKey key = makeCacheKey(a.id, b.id, IV3{0, 0, 0}, IV3{0, 0, 0}, rp, rr);
                    const size_t cap = w.cache.e.size();
                    size_t idx = (size_t)(key.hash() % cap);
                    const CacheValue<float>* hit = nullptr;
                    for (size_t p = 0; p < std::min<size_t>(cap, 16); ++p) {
                        const auto& en = w.cache.e[idx];
                        if (!en.valid) break;
                        if (en.key == key) {
                            hit = &en.value;
                            break;
                        }
                        idx = (idx + 1) % cap;
                    }
                    if (hit) {
                        hits++;
                        if (hit->has_collision) {
                            Manifold<float> m;
                            m.a = a.id;
                            m.b = b.id;
                            m.friction = std::sqrt(a.friction * b.friction);
                            m.restitution = fmx(a.restitution, b.restitution);
                            for (uint32_t i = 0; i < hit->n; ++i) m.addContact(hit->c[i]);
                            out[(size_t)t].push_back(m);
                        }
                        continue;
                    }
                    misses++;
                }
                DetectResult<float> r = detectVoxelCollisions(a, ca, b, cb, nullptr, 0);
                if (r.has_collision) out[(size_t)t].push_back(r.m);
            }
        });
    }
    for (auto& x : th) x.join();
    int contacts = 0;
    for (auto& v : out)
        for (auto& m : v) {
            contacts += (int)m.n;
            w.cm.addManifold(m);
        }
    w.stats.cache_hits = (uint32_t)hits.load();
    w.stats.cache_misses = (uint32_t)misses.load();
    w.stats.manifolds = (uint32_t)w.cm.cur.size();
    return contacts;
}

int vxo_narrow_phase_threaded(void* p, const vxp_pair* pairs, uint32_t n, int threads) {
    if (prec(p) != 32) return VXP_ERR_ARG;
    return narrow_threaded(H<float>(p)->w, pairs, n, threads);
}

// One VoxelPhysicsSystem.step with enable_threading: threaded narrow phase,
// then the (single-threaded) solve and the sleep update.
int vxo_step_threaded(void* p, float dt, const vxp_pair* pairs, uint32_t n, int threads) {
    if (prec(p) != 32) return VXP_ERR_ARG;
    World<float>& w = H<float>(p)->w;
    w.stats = Stats{};
    w.stats.pairs_in = n;
    if (w.wcfg.enable_sleeping && w.allDynamicSleeping()) {
        w.stats.step_skipped = 1;
        return 0;
    }
    narrow_threaded(w, pairs, n, threads);
    w.solve(dt);
    if (w.wcfg.enable_sleeping)
        for (auto& b : w.bodies)
            if (b.type == B_DYNAMIC && !b.sleeping) b.updateSleepState(dt);
    return 0;
}

int vxo_mass_properties(float vs, const vxp_brick* bricks, uint32_t n, float density, float* inv_mass,
                        float* inv_I) {
    std::vector<IV3> pos(n);
    std::vector<uint8_t> vox((size_t)n * 512);
    for (uint32_t i = 0; i < n; ++i) {
        pos[i] = {bricks[i].pos[0], bricks[i].pos[1], bricks[i].pos[2]};
        std::memcpy(&vox[(size_t)i * 512], bricks[i].voxels, 512);
    }
    Collider<float> c;
    if (!c.build(vs, pos.data(), vox.data(), n)) return VXP_ERR_ARG;
    float im;
    M3<float> I;
    computeMassProperties(c, density, &im, &I);
    *inv_mass = im;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) inv_I[i * 3 + j] = I.m[i][j];
    return 0;
}

// Collider metadata: min_bound[3], max_bound[3], local_aabb min[3] max[3], solid_count.
int vxo_collider_metadata(float vs, const vxp_brick* bricks, uint32_t n, int32_t* bounds6, float* aabb6,
                          uint32_t* solid) {
    std::vector<IV3> pos(n);
    std::vector<uint8_t> vox((size_t)n * 512);
    for (uint32_t i = 0; i < n; ++i) {
        pos[i] = {bricks[i].pos[0], bricks[i].pos[1], bricks[i].pos[2]};
        std::memcpy(&vox[(size_t)i * 512], bricks[i].voxels, 512);
    }
    Collider<float> c;
    if (!c.build(vs, pos.data(), vox.data(), n)) return VXP_ERR_ARG;
    bounds6[0] = c.min_bound.x; bounds6[1] = c.min_bound.y; bounds6[2] = c.min_bound.z;
    bounds6[3] = c.max_bound.x; bounds6[4] = c.max_bound.y; bounds6[5] = c.max_bound.z;
    aabb6[0] = c.local_aabb.mn.x; aabb6[1] = c.local_aabb.mn.y; aabb6[2] = c.local_aabb.mn.z;
    aabb6[3] = c.local_aabb.mx.x; aabb6[4] = c.local_aabb.mx.y; aabb6[5] = c.local_aabb.mx.z;
    *solid = c.solid_count;
    return 0;
}

// ---- known-answer helpers (reference unit tests) --------------------------
uint8_t vxo_classify(int solid, uint8_t empty_mask) { return classifyVoxel(solid != 0, empty_mask); }
uint8_t vxo_classify_from_neighbors(int solid, int nx, int px, int ny, int py, int nz, int pz) {
    return classifyFromNeighbors(solid != 0, nx, px, ny, py, nz, pz);
}
uint8_t vxo_compute_normal_index(uint8_t m) { return computeNormalIndex(m); }
uint8_t vxo_find_closest_normal(float x, float y, float z) { return findClosestNormalIndex(V3<float>{x, y, z}); }
void vxo_normal_vec(uint8_t idx, float* out) {
    const V3<float> v = getNormalVec3<float>(idx);
    out[0] = v.x; out[1] = v.y; out[2] = v.z;
}
int vxo_should_collide(uint8_t ta, uint8_t tb) { return shouldCheckCollision(ta, tb) ? 1 : 0; }
uint64_t vxo_feature_id(const int32_t* a, const int32_t* b) {
    return computeFeatureId(IV3{a[0], a[1], a[2]}, IV3{b[0], b[1], b[2]});
}
void vxo_brick_coords(const int32_t* v, int32_t* brick, int32_t* local) {
    brick[0] = divFloor8(v[0]); brick[1] = divFloor8(v[1]); brick[2] = divFloor8(v[2]);
    local[0] = mod8(v[0]); local[1] = mod8(v[1]); local[2] = mod8(v[2]);
}
int vxo_sat_early_out(const float* a, const float* b) { return satEarlyOut(obbIn(a), obbIn(b)) ? 1 : 0; }
int vxo_sat_with_penetration(const float* a, const float* b, float* depth, float* axis) {
    V3<float> ax;
    float d;
    if (!satWithPenetration(obbIn(a), obbIn(b), &ax, &d)) return 0;
    *depth = d;
    axis[0] = ax.x; axis[1] = ax.y; axis[2] = ax.z;
    return 1;
}
void vxo_soft_params(float hz, float zeta, float h, float* out) {
    const SoftParams<float> s = computeSoftParams(hz, zeta, h);
    out[0] = s.bias_rate; out[1] = s.mass_coeff; out[2] = s.impulse_coeff;
}
void vxo_compute_orthogonal(const float* v, float* out) {
    const V3<float> r = computeOrthogonal(V3<float>{v[0], v[1], v[2]});
    out[0] = r.x; out[1] = r.y; out[2] = r.z;
}
void vxo_integrate_rotation_small(const float* q, const float* d, float* out) {
    const Q<float> r = integrateRotationSmall(Q<float>{q[0], q[1], q[2], q[3]}, V3<float>{d[0], d[1], d[2]});
    out[0] = r.x; out[1] = r.y; out[2] = r.z; out[3] = r.w;
}
void vxo_integrate_rotation(const float* q, const float* w, float dt, float* out) {
    const Q<float> r = integrateRotation(Q<float>{q[0], q[1], q[2], q[3]}, V3<float>{w[0], w[1], w[2]}, dt);
    out[0] = r.x; out[1] = r.y; out[2] = r.z; out[3] = r.w;
}
void vxo_from_axis_angle(const float* axis, float angle, float* out) {
    const Q<float> r = fromAxisAngle(V3<float>{axis[0], axis[1], axis[2]}, angle);
    out[0] = r.x; out[1] = r.y; out[2] = r.z; out[3] = r.w;
}
void vxo_transform_point(const float* pos, const float* q, const float* p, float* out) {
    const Xf<float> t{{pos[0], pos[1], pos[2]}, {q[0], q[1], q[2], q[3]}};
    const V3<float> r = transformPoint(t, V3<float>{p[0], p[1], p[2]});
    out[0] = r.x; out[1] = r.y; out[2] = r.z;
}
void vxo_inverse_transform_point(const float* pos, const float* q, const float* p, float* out) {
    const Xf<float> t{{pos[0], pos[1], pos[2]}, {q[0], q[1], q[2], q[3]}};
    const V3<float> r = inverseTransformPoint(t, V3<float>{p[0], p[1], p[2]});
    out[0] = r.x; out[1] = r.y; out[2] = r.z;
}
void vxo_quat_rotate(const float* q, const float* v, float* out) {
    const V3<float> r = qrotate(Q<float>{q[0], q[1], q[2], q[3]}, V3<float>{v[0], v[1], v[2]});
    out[0] = r.x; out[1] = r.y; out[2] = r.z;
}
void vxo_mat3_inverse(const float* m, float* out) {
    M3<float> a;
    for (int i = 0; i < 9; ++i) a.m[i / 3][i % 3] = m[i];
    const M3<float> r = minverse(a);
    for (int i = 0; i < 9; ++i) out[i] = r.m[i / 3][i % 3];
}
// VoxelBody.getWorldInvInertia (body.zig:386-392) of a dynamic body with
// rotation q and local inverse inertia inv_local (row-major 3x3).
void vxo_world_inv_inertia(const float* q, const float* inv_local, float* out) {
    Body<float> b;
    b.type = B_DYNAMIC;
    b.inv_mass = 1.0f;
    b.rot = Q<float>{q[0], q[1], q[2], q[3]};
    for (int i = 0; i < 9; ++i) b.inv_I_local.m[i / 3][i % 3] = inv_local[i];
    const M3<float> r = b.worldInvInertia();
    for (int i = 0; i < 9; ++i) out[i] = r.m[i / 3][i % 3];
}
float vxo_sinf(float x) { return sincos_f32(x, 0); }
float vxo_cosf(float x) { return sincos_f32(x, 1); }

// Sequential ContactManifold.addContact over n contacts (pens, feature ids);
// writes, per slot, the index of the input contact it holds.
int vxo_manifold_replay(const float* pens, const uint64_t* fids, uint32_t n, uint32_t* slots, uint32_t* n_out) {
    Manifold<float> m;
    for (uint32_t i = 0; i < n; ++i) {
        Contact<float> c;
        c.penetration = pens[i];
        c.feature_id = fids[i];
        c.point.x = (float)i;  // carry the input index through the copy
        m.addContact(c);
    }
    for (uint32_t s = 0; s < m.n; ++s) slots[s] = (uint32_t)m.c[s].point.x;
    *n_out = m.n;
    return 0;
}

// ContactManager warm-start known answer (narrow_phase.zig:1796-1825): add a
// manifold with one contact (feature id, impulse), beginFrame, add a second
// one; returns the transferred impulse of the first contact.
float vxo_contact_manager_warm(uint64_t fid1, float impulse1, uint64_t fid2) {
    ContactManager<float> cmg;
    Manifold<float> m1;
    m1.a = 1; m1.b = 2;
    Contact<float> c1;
    c1.feature_id = fid1;
    c1.normal_impulse = impulse1;
    m1.addContact(c1);
    cmg.addManifold(m1);
    cmg.beginFrame();
    Manifold<float> m2;
    m2.a = 1; m2.b = 2;
    Contact<float> c2;
    c2.feature_id = fid2;
    m2.addContact(c2);
    cmg.addManifold(m2);
    return cmg.cur[0].c[0].normal_impulse;
}

// Brick-pair cache known answers.
void* vxo_cache_create(uint32_t cap) { return new BrickPairCache<float>(cap); }
void vxo_cache_destroy(void* c) { delete static_cast<BrickPairCache<float>*>(c); }
static CacheKey cacheKeyIn(const uint32_t* ids, const float* rel_pos, const float* rel_rot) {
    return makeCacheKey(ids[0], ids[1], IV3{0, 0, 0}, IV3{0, 0, 0}, V3<float>{rel_pos[0], rel_pos[1], rel_pos[2]},
                        Q<float>{rel_rot[0], rel_rot[1], rel_rot[2], rel_rot[3]});
}
int vxo_cache_get(void* c, const uint32_t* ids, const float* rel_pos, const float* rel_rot, uint32_t* contact_count) {
    auto* k = static_cast<BrickPairCache<float>*>(c);
    const CacheValue<float>* v = k->get(cacheKeyIn(ids, rel_pos, rel_rot));
    if (!v) return 0;
    *contact_count = v->n;
    return v->has_collision ? 2 : 1;
}
void vxo_cache_put(void* c, const uint32_t* ids, const float* rel_pos, const float* rel_rot, int has_collision,
                   uint32_t contact_count) {
    auto* k = static_cast<BrickPairCache<float>*>(c);
    CacheValue<float> v;
    v.has_collision = has_collision != 0;
    v.n = (uint8_t)contact_count;
    k->put(cacheKeyIn(ids, rel_pos, rel_rot), v);
}
void vxo_cache_invalidate(void* c, uint32_t id) { static_cast<BrickPairCache<float>*>(c)->invalidateBody(id); }
void vxo_cache_begin_frame(void* c) { static_cast<BrickPairCache<float>*>(c)->beginFrame(); }
void vxo_cache_stats(void* c, uint64_t* out4) {
    auto* k = static_cast<BrickPairCache<float>*>(c);
    out4[0] = k->hits; out4[1] = k->misses; out4[2] = k->evictions; out4[3] = k->invalidations;
}
int vxo_cache_key_eq(const uint32_t* ids1, const float* p1, const float* r1, const uint32_t* ids2, const float* p2,
                     const float* r2) {
    return cacheKeyIn(ids1, p1, r1) == cacheKeyIn(ids2, p2, r2) ? 1 : 0;
}

// GraphColoring.build known answer over (a, b) manifold pairs.
int vxo_graph_colouring(const uint32_t* ab, uint32_t n, uint8_t* colours) {
    std::vector<Manifold<float>> ms(n);
    for (uint32_t i = 0; i < n; ++i) {
        ms[i].a = ab[2 * i];
        ms[i].b = ab[2 * i + 1];
    }
    uint32_t mx = 0;
    auto c = graphColouring(ms, &mx);
    for (uint32_t i = 0; i < n; ++i) colours[i] = c[i];
    return (int)mx + 1;
}

// VoxelBody.updateSleepState known answer: steps a resting dynamic body n times.
int vxo_sleep_after(uint32_t n, float dt) {
    Body<float> b;
    for (uint32_t i = 0; i < n; ++i) b.updateSleepState(dt);
    return b.sleeping ? 1 : 0;
}

uint32_t vxo_jp_priority(uint32_t k) { return jpPriority(k); }

}  // extern "C"
