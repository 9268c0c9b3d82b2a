"""IslandManager (src/islands.zig:25-495) in the oracle, the checker the
device's island statistics are compared with.

* The reference's own island tests, restated: "IslandManager build islands"
  (islands.zig:785-816), "buildIslandsWithBodyTypes isolates bodies through
  static" (islands.zig:857-888), and the union-find chain of "UnionFind path
  compression" (islands.zig:769-783) as one island of 100 bodies.
* The oracle's per-step island statistics on the 64-cube scene against an
  independent restatement written here from the reference's rules: islands
  are the connected components of the manifold graph without static bodies,
  rebuilt when the frame's manifold pair-key sequence changes; an island
  sleeps after its bodies have been still for 0.5 s (timers in f32), the body
  for island body id k being the k-th body of the table.
"""
import numpy as np
import pytest

import oracle_api as O

STATIC, DYNAMIC = 0, 2


def test_build_islands_kat():
    isl, total, largest = O.islands_kat([(0, 1), (1, 2), (3, 4)], 5)
    assert total == 2 and largest == 3
    assert (isl[:5] >= 0).all()
    assert isl[0] == isl[1] == isl[2]
    assert isl[3] == isl[4]
    assert isl[0] != isl[3]


def test_static_bodies_isolate_islands_kat():
    isl, total, _ = O.islands_kat([(0, 1), (0, 2), (2, 3)], 4, types=[STATIC, DYNAMIC, DYNAMIC, DYNAMIC])
    assert isl[2] == isl[3]
    assert isl[1] != isl[2]
    assert isl[0] not in (isl[1], isl[2])  # the static body is an island of its own
    assert total == 3


def test_union_find_chain_kat():
    isl, total, largest = O.islands_kat([(i - 1, i) for i in range(1, 100)], 100)
    assert total == 1 and largest == 100
    assert (isl == isl[0]).all()


def test_empty_manifold_list_has_no_islands():
    isl, total, largest = O.islands_kat([], 4)
    assert total == 0 and largest == 0 and (isl == -1).all()


class IslandModel:
    """The reference's island rules restated from islands.zig in Python."""

    def __init__(self):
        self.prev_keys = None
        self.dirty = True
        self.islands = []  # list of (set of body ids), parallel to timers / asleep
        self.timers = []
        self.asleep = []

    def step(self, manifolds, bodies, dt):
        keys = [(int(min(a, b)), int(max(a, b))) for a, b in zip(manifolds["body_a_id"], manifolds["body_b_id"])]
        if self.dirty or keys != self.prev_keys or not self.islands:
            self.dirty = False
            self.prev_keys = keys
            typ = {int(i): int(t) for i, t in zip(bodies["id"], bodies["body_type"])}
            parent = {}

            def find(x):
                while parent.setdefault(x, x) != x:
                    x = parent[x]
                return x

            ids = set()
            for a, b in keys:
                ids.update((a, b))
                if typ[a] != STATIC and typ[b] != STATIC:
                    ra, rb = find(a), find(b)
                    if ra != rb:
                        parent[max(ra, rb)] = min(ra, rb)
            comps = {}
            for i in ids:
                comps.setdefault(find(i), set()).add(i)
            self.islands = list(comps.values())
            self.timers = [np.float32(0)] * len(self.islands)
            self.asleep = [False] * len(self.islands)
        thr = np.float32(0.1) * np.float32(0.1)
        for k, members in enumerate(self.islands):
            still = True
            for bid in members:
                if bid >= len(bodies) or bodies["body_type"][bid] != DYNAMIC:
                    continue
                v = bodies["linear_velocity"][bid].astype(np.float32)
                w = bodies["angular_velocity"][bid].astype(np.float32)
                lv = (v[0] * v[0] + v[1] * v[1]) + v[2] * v[2]
                lw = (w[0] * w[0] + w[1] * w[1]) + w[2] * w[2]
                if lv > thr or lw > thr:
                    still = False
                    break
            if still:
                self.timers[k] = np.float32(self.timers[k] + np.float32(dt))
                if self.timers[k] >= np.float32(0.5):
                    self.asleep[k] = True
            else:
                self.timers[k] = np.float32(0)
                self.asleep[k] = False
        n = len(self.islands)
        return n, sum(self.asleep), max((len(m) for m in self.islands), default=0)


@pytest.mark.parametrize("scene", ["config1", "basic"])
def test_oracle_island_stats_follow_the_reference_rules(vxp, scene):
    """The 64-cube scene (contacts change every few steps: islands rebuild
    and seldom sleep) and the reference's example scene (one box comes to
    rest on the slab: the graph stops changing and islands sleep)."""
    if scene == "config1":
        sc = vxp.scenes.config1(mass_fn=O.mass_fn, seed=3)
    else:
        sc = vxp.scenes.basic_example(O.mass_fn)
    r = O.OracleWorld()
    r.load_scene(sc)
    model = IslandModel()
    dt = np.float32(sc.dt)
    seen_sleep = seen_islands = 0
    for s in range(240):
        before = r.get_bodies()  # island sleep reads the velocities before the solve
        r.step(dt)
        st = r.stats()
        if st["step_skipped"]:
            assert st["island_count"] == 0
            continue
        n, asleep, largest = model.step(r.manifolds(), before, dt)
        assert (st["island_count"], st["sleeping_islands"], st["largest_island_size"]) == (n, asleep, largest), s
        assert st["active_islands"] == n - asleep
        seen_islands += n > 0
        seen_sleep += asleep > 0
    r.close()
    assert seen_islands > 20
    if scene == "basic":
        assert seen_sleep > 0
