"""Per-substep parity: every body's position, rotation and velocities after
each substep (before the position sweeps and writeBack), device against the
oracle, with the reference's own colouring (GraphColoring.build order) and
with the project colouring, in both launch modes (and the cluster sweeps).  Bit for bit; the 1e-5
relative bound of the float results is asserted too, for the record."""
import numpy as np
import pytest

import oracle_api as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode,solver", [(0, None), (1, 1), (1, 2)])
@pytest.mark.parametrize("colouring", [1, 0])
def test_substep_states_match_oracle(vxp, mode, solver, colouring):
    sc = vxp.scenes.config1(O.mass_fn)
    cfg = dict(substeps=4, colouring=colouring)
    g = vxp.VoxelPhysicsSystem(**cfg)
    g.load_scene(sc)
    g.set_launch_mode(mode)
    if solver is not None:
        g.set_solver_mode(solver)
    g.set_substep_record(True)
    r = O.OracleWorld(**cfg)
    r.load_scene(sc)
    r.set_substep_record(True)
    dt = np.float32(sc.dt)
    recorded = 0
    for s in range(80):
        pairs = r.pairs()
        g.step(dt, pairs)
        r.step(dt, pairs)
        gs, rs = g.substeps(), r.substeps()
        assert gs.shape == rs.shape, f"step {s}: {gs.shape} vs {rs.shape}"
        if gs.size:
            rel = np.abs(gs.astype(np.float64) - rs) / np.maximum(np.abs(rs.astype(np.float64)), 1.0)
            assert rel.max() <= 1e-5, f"step {s}: relative difference {rel.max()}"
            assert gs.tobytes() == rs.tobytes(), f"step {s}: substep states differ"
            recorded += gs.shape[0]
    assert recorded >= 4 * 40
    g.close()
    r.close()
