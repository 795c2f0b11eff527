"""The bounded device-side waits' time-out paths, made to run by ASD_FLAG_WAIT_TIMEOUT (each wait for
a block's bulk copies gives up at once).  No wait is left unbounded and nothing faults: a timed-out
block of the stage kernel reads its exchange words and neighbour spins from global memory instead
of shared memory, so the spins still match the oracle, and waits again (bounded) before retiring
so no copy lands in a retired block; a timed-out block of the x transform leaves its tile and the
long-range field of that evaluation is flagged invalid.  Either way asd_sync reports
ASD_ETIMEOUT once and clears it, and the handle and the context stay usable."""
import numpy as np
import pytest

import asd_b200 as A
import asd_lattice as LT
from helpers import maxdiff
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("staging", [1, 2])
def test_stage_staging_wait_times_out_and_falls_back(gpu, staging):
    s = LT.sc_ferromagnet(16)
    S0 = LT.random_spins(s.nspins, 0)
    o = O.Oracle(s)
    o.set_spins(S0)
    o.step(100)
    with A.Handle(A.RunParams(precision=A.FP32, flags=A.FLAG_COMPENSATED | A.FLAG_WAIT_TIMEOUT), s) as h:
        h.set_launch_shape(256, staging)
        h.set_spins(S0)
        h.step(100)
        with pytest.raises(A.AsdError) as ex:
            h.sync()
        assert ex.value.code == A.ASD_ETIMEOUT
        assert "staging wait" in str(ex.value)
        h.sync()                                   # reported once, then cleared
        g = h.get_spins()
    assert maxdiff(g, o.spins()) <= 1e-5, maxdiff(g, o.spins())


def test_transform_wait_times_out_and_context_stays_usable(gpu):
    s = LT.sc_ferromagnet((8, 8, 8), pbc=(0, 0, 0), dipole=True)
    S0 = LT.random_spins(s.nspins, 1)
    with A.Handle(A.RunParams(precision=A.FP32, flags=A.FLAG_COMPENSATED | A.FLAG_WAIT_TIMEOUT), s) as h:
        assert "plane kernels" in h.tuning()
        h.set_spins(S0)
        h.step(2)
        with pytest.raises(A.AsdError) as ex:
            h.sync()
        assert ex.value.code == A.ASD_ETIMEOUT
        assert "long-range" in str(ex.value)
    # a new handle on the same device runs normally and matches the oracle
    o = O.Oracle(s)
    o.set_spins(S0)
    o.step(20)
    with A.Handle(A.RunParams(precision=A.FP32, flags=A.FLAG_COMPENSATED), s) as h:
        h.set_spins(S0)
        h.step(20)
        h.sync()
        g = h.get_spins()
    assert maxdiff(g, o.spins()) <= 1e-5, maxdiff(g, o.spins())
