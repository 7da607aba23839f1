"""Ensemble of independent runs (batched execution on one GPU): every member
ends in the same state as the same run alone (deterministic deposit)."""
import numpy as np
import pytest

from gample_b200 import capi
from tests.helpers import condition

KEY = ["x", "y", "vx", "vy", "vz", "piflag"]


def _members():
    out = []
    for i, (n, order, ppc, bz) in enumerate([(32, 1, 16, 0.0), (48, 3, 24, 0.02), (64, 5, 16, 0.05),
                                             (40, 3, 32, 0.01)]):
        c = condition(ngx=n, ngy=n, order=order, ppc=ppc, xbc="Dirichlet", ybc="periodic", bz_tesla=bz,
                      deposit_mode=1, end=6)
        out.append(c)
    return out


@pytest.mark.gpu
def test_ensemble_members_equal_the_runs_alone(gpu):
    conds = _members()
    ens = capi.Ensemble(conds, threads=4)
    ens.initialize()
    ens.run(4)
    ms = ens.time_cycles(2)  # the same cycles, timed on the device
    assert ms > 0.0
    got = [[np.sort(m.particles(s), order=KEY) for s in range(2)] for m in ens.members]
    fields = [m.field("Ex") for m in ens.members]
    ens.close()
    for k, c in enumerate(conds):
        sim = capi.Sim(c)
        sim.initialize()
        sim.run(6)
        for s in range(2):
            np.testing.assert_array_equal(np.sort(sim.particles(s), order=KEY), got[k][s])
        np.testing.assert_array_equal(sim.field("Ex"), fields[k])
        sim.close()
