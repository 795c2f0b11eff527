"""The applied field changed between steps, as the reference's field ramp sets llg::applied
before each llg::integrate call (src/ramp_field.cpp:221-223), through every route that carries
it to the device: single-step calls (the one-step graph's first node takes it as a kernel
parameter), multi-step calls and field reads (an update launched before the work when a
single-step call has not yet carried it), two updates in a row, and a mix, against the FP64
oracle given the same field before each step.

Tolerances as in test_gpu_parity: FP64 plain bit-exact, fused FP64 1e-10, FP32 1e-5."""
import numpy as np
import pytest

import asd_b200 as A
import asd_lattice as LT
from helpers import maxdiff
from oracle import oracle as O

pytestmark = pytest.mark.gpu

# (fields set before the call, the last one in effect; steps; read the field before stepping)
SEQUENCE = [
    ([(0.0, 0.0, 0.5)], 1, False),
    ([(0.2, 0.0, 0.5)], 3, False),
    ([(0.2, -0.1, 0.4)], 1, False),
    ([(0.0, 0.3, 0.0), (1.0, 0.0, -0.2)], 1, False),
    ([(0.4, 0.1, 0.1)], 1, True),
    ([(0.4, 0.1, 0.1)], 2, False),
    ([(-0.3, 0.2, 0.6)], 1, True),
    ([(0.1, 0.1, 0.1)], 1, False),
]

TOL = {A.FP64_PLAIN: 0.0, A.FP64_FUSED: 1e-10, A.FP32: 1e-5}


@pytest.mark.parametrize("prec", [A.FP64_PLAIN, A.FP64_FUSED, A.FP32])
def test_applied_field_between_steps_matches_oracle(gpu, prec):
    s = LT.sc_ferromagnet(8, T=50.0)
    S0 = LT.random_spins(s.nspins, 4)
    flags = A.FLAG_COMPENSATED if prec == A.FP32 else 0
    o = O.Oracle([s], integrator=A.HEUN, dt=1e-16, seed=1)
    o.set_spins(S0)
    with A.Handle(A.RunParams(precision=prec, flags=flags, seed=1), [s]) as h:
        h.set_spins(S0)
        for fields, steps, read in SEQUENCE:
            for b in fields:
                h.set_applied(b)
            o.set_applied(fields[-1])
            if read:                                   # a field read between the update and the step
                f = h.get_field()
                assert np.all(np.isfinite(f))
            h.step(steps)
            o.step(steps)
            g = h.get_spins()
            err = maxdiff(g, o.spins())
            if prec == A.FP64_PLAIN:
                assert np.array_equal(g, o.spins()), (fields, steps, err)
            else:
                assert err <= TOL[prec], (fields, steps, err)
