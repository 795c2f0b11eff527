"""Bitwise checkpoint and restart (the reference's restart path, src/spins.cpp:342-398, reads the
spins back from text and renormalises them; asd_get_state / asd_set_state carry the exact state):
a run stopped at step k, its state restored into a new handle, continues bit for bit like the
uninterrupted run, for every arithmetic form, at T = 0 and T > 0 (the thermal draws are keyed on
the step), with the dipole field and with the two-temperature model."""
import numpy as np
import pytest

import asd_b200 as A
import asd_lattice as LT

pytestmark = pytest.mark.gpu

TTM = dict(gamma_e=3.0e3, Cl=2.0e6, G_ep=1.0e17, pump_time=2e-15, pump_fluence=4e21, cooling_time=1e-12,
           initial_T=40.0, pulses=[(1.0, 3e-15), (0.5, 6e-15)])


def resumed_equals_uninterrupted(systems, params, k, m, ttm=False):
    n = sum(s.nspins for s in systems)
    S0 = LT.random_spins(n, 0)
    with A.Handle(params, systems) as h:
        h.set_spins(S0)
        if ttm:
            h.set_ttm(**TTM)
        h.step(k + m)
        want = h.get_spins()
    with A.Handle(params, systems) as h:
        h.set_spins(S0)
        if ttm:
            h.set_ttm(**TTM)
        h.step(k)
        state = h.get_state()
    with A.Handle(params, systems) as h:
        if ttm:
            h.set_ttm(**TTM)
        h.set_state(state)
        assert h.get_step() == k
        h.step(m)
        got = h.get_spins()
    assert np.array_equal(got, want), float(np.abs(got - want).max())


@pytest.mark.parametrize("prec", [A.FP64_PLAIN, A.FP32, A.FP64_FUSED])
@pytest.mark.parametrize("T", [0.0, 300.0])
def test_restart_bitwise(gpu, prec, T):
    s = LT.bct2_antiferromagnet(4, T=T)
    p = A.RunParams(precision=prec, flags=A.FLAG_COMPENSATED if prec == A.FP32 else 0, seed=3)
    resumed_equals_uninterrupted([s], p, 37, 45)


@pytest.mark.parametrize("prec", [A.FP32, A.FP64_FUSED, A.FP64_PLAIN])
def test_restart_bitwise_dipole(gpu, prec):
    s = LT.sc_ferromagnet((8, 8, 8), pbc=(0, 0, 0), dipole=True)
    p = A.RunParams(precision=prec, flags=A.FLAG_COMPENSATED if prec == A.FP32 else 0, update=1)
    resumed_equals_uninterrupted([s], p, 33, 20)


def test_restart_bitwise_ttm_replicas(gpu):
    reps = [LT.sc_ferromagnet(4, T=10.0, stream=0), LT.sc_ferromagnet(5, T=10.0, stream=1)]
    p = A.RunParams(precision=A.FP32, flags=A.FLAG_COMPENSATED, seed=5)
    resumed_equals_uninterrupted(reps, p, 40, 40, ttm=True)


def test_state_is_checked(gpu):
    s = LT.sc_ferromagnet(4)
    with A.Handle(A.RunParams(precision=A.FP32, flags=A.FLAG_COMPENSATED), s) as h:
        st = h.get_state()
    with A.Handle(A.RunParams(precision=A.FP64_FUSED), s) as h:
        with pytest.raises(A.AsdError):
            h.set_state(st)
    with A.Handle(A.RunParams(precision=A.FP32, flags=A.FLAG_COMPENSATED), LT.sc_ferromagnet(5)) as h:
        with pytest.raises(A.AsdError):
            h.set_state(st)
        with pytest.raises(A.AsdError):
            h.set_state(b"XXXX" + st[4:])
