"""Failure detection on the device, in the forms that fault no GPU.

* A bounded wait that runs out: the grid barrier's wait limit is set to a
  few nanoseconds, so a real grid-launched step gives up at its first uneven
  barrier.  The call must report VXP_ERR_TIMEOUT, every kernel must return,
  and the same context must step on afterwards, bit-exact with the oracle.
* Corrupted state injected from the host: NaN in a body's pose or velocity
  must come back as `BodyState.writeBack` resets it (src/solver.zig:249-259:
  the body's last finite position, else (0, 2, 0); identity rotation; zero
  velocities), exactly as the oracle does.
"""
import numpy as np
import pytest

import oracle_api as O
from test_gpu_parity import _first_diff

pytestmark = pytest.mark.gpu


def _step_both(g, r, dt, n):
    for s in range(n):
        pairs = r.pairs()
        g.step(dt, pairs)
        r.step(dt, pairs)
        gb, rb = g.get_bodies(), r.get_bodies()
        assert gb.tobytes() == rb.tobytes(), f"step {s}: bodies differ in {_first_diff(gb, rb)}"


def test_wait_limit_runs_out_and_the_context_recovers(vxp):
    """Grid launch of a 216-box pile with warm starting, the brick-pair cache
    and sleeping off, so that a step depends on the bodies alone and a step
    abandoned half-way leaves nothing the next one reads: 10 steps in
    lockstep, one step with a 1 ns barrier wait (VXP_ERR_TIMEOUT), then the
    default limit, the bodies set back to the oracle's, and 10 more steps
    bit-exact."""
    cfg = dict(substeps=8, enable_warm_starting=0, warm_starting=0, use_brick_pair_cache=0, enable_sleeping=0)
    sc = vxp.scenes.config2(mass_fn=O.mass_fn, n_side=6, seed=41)
    g = vxp.VoxelPhysicsSystem(**cfg)
    g.load_scene(sc)
    g.set_launch_mode(1)  # cooperative grid: the kernels with bounded barriers
    r = O.OracleWorld(**cfg)
    r.load_scene(sc)
    dt = np.float32(sc.dt)
    for _ in range(240):  # let the lowest layers land, so the step has uneven work
        r.step(dt)
    g.set_bodies(r.get_bodies())
    _step_both(g, r, dt, 10)

    g.set_wait_limit_ns(1)
    with pytest.raises(vxp.system.VxpError) as err:
        g.step(dt, r.pairs())
        g.synchronize()
        g.get_bodies()
    assert err.value.code == vxp.abi.VXP_ERR_TIMEOUT, str(err.value)
    assert "ran out" in str(err.value)

    g.set_wait_limit_ns(0)
    g.set_bodies(r.get_bodies())
    _step_both(g, r, dt, 10)
    g.close()
    r.close()


def test_nan_state_is_reset_like_write_back(vxp):
    """A 64-box pile (config-2 shapes, 2.8 m lattice) while the boxes still
    fall: one body gets a NaN position, and two bodies without a contact a NaN
    linear velocity and a NaN angular velocity.  After a
    step, device and oracle agree bit for bit, and the three bodies carry the
    reset of BodyState.writeBack (a NaN angular velocity fails
    integrateRotation's small-angle test, src/math.zig:755-768, and turns the
    rotation into NaN too)."""
    sc = vxp.scenes.config2(mass_fn=O.mass_fn, n_side=4, seed=43)
    g = vxp.VoxelPhysicsSystem(substeps=8)
    g.load_scene(sc)
    r = O.OracleWorld(substeps=8)
    r.load_scene(sc)
    dt = np.float32(sc.dt)
    _step_both(g, r, dt, 3)
    b = r.get_bodies()
    start = b.copy()
    # bodies that get no contact this step (a fresh oracle's narrow phase on
    # the same bodies and pairs), so no impulse carries their NaN elsewhere;
    # a NaN position drops out of the pair list by itself
    probe = O.OracleWorld(substeps=8)
    probe.load_scene(sc)
    probe.set_bodies(b)
    probe.narrow_phase(r.pairs())
    touching = {int(x) for m in probe.manifolds() if m["contact_count"] for x in (m["body_a_id"], m["body_b_id"])}
    probe.close()
    free = [i for i in range(3, len(b)) if int(b["id"][i]) not in touching]
    assert len(free) >= 2, len(free)
    i_pos, i_lin, i_ang = 2, free[0], free[-1]
    nan = np.float32(np.nan)
    b["position"][i_pos] = (nan, nan, nan)
    b["linear_velocity"][i_lin][1] = nan
    b["angular_velocity"][i_ang][2] = nan
    g.set_bodies(b)
    r.set_bodies(b)
    _step_both(g, r, dt, 1)
    out = g.get_bodies()
    for i in (i_pos, i_lin, i_ang):
        assert np.all(np.isfinite(out["position"][i])), i
        assert tuple(out["rotation"][i]) == (0.0, 0.0, 0.0, 1.0), i
        assert not np.any(out["linear_velocity"][i]) and not np.any(out["angular_velocity"][i]), i
    # NaN position: no finite position to go back to, so (0, 2, 0)
    assert tuple(out["position"][i_pos]) == (0.0, 2.0, 0.0)
    # NaN velocity: back to the position the step started from
    assert out["position"][i_lin].tobytes() == start["position"][i_lin].tobytes()
    assert out["position"][i_ang].tobytes() == start["position"][i_ang].tobytes()
    _step_both(g, r, dt, 5)
    g.close()
    r.close()
