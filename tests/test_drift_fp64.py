"""FP32 against an FP64 replay of the same solver (the oracle in both
precisions; the device path is bit-identical to the FP32 oracle).  The first
steps, before contacts amplify differences, stay within the 1e-5 relative
tolerance of the device path's float results."""
import numpy as np

import oracle_api as O
from drift_report import drift


def test_first_steps_within_tolerance(vxp):
    sc = vxp.scenes.config1(O.mass_fn)
    rows = drift(sc, 5, np.float32(sc.dt), substeps=4)
    for r in rows:
        assert r["max_rel_dx"] <= 1e-5, r
        assert r["max_dv"] <= 1e-4, r
    assert np.isfinite([r["max_dx"] for r in rows]).all()
