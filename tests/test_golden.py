"""The oracle against its committed golden fixtures (tests/golden/): config
1's body table after steps 1, 10, 50, 150, 300 and its manifolds after step
20, bit for bit.  The fixtures come from tests/golden/make_golden.py."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_golden  # noqa: E402


def test_oracle_reproduces_golden_fixtures(vxp):
    snaps, man = make_golden.config1_run(vxp)
    gold = np.load(os.path.join(HERE, "golden", "config1_bodies.npz"))
    assert sorted(gold.files) == sorted(snaps)
    for k in gold.files:
        assert gold[k].tobytes() == snaps[k].tobytes(), k
    gman = np.load(os.path.join(HERE, "golden", "config1_manifolds.npy"))
    assert gman.tobytes() == man.tobytes()
