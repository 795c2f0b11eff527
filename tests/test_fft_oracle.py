"""Pins of the FFT restatement (oracle/fft_oracle.py) that the CPU baseline and the bench's
reference arm time on the sc 128x128x64 dipole lattice: its lattice builder against the reference's own
CSR assembly and the library's builder, and its FFT long-range field and Heun step against the
direct-sum oracle (oracle/asd_oracle.c)."""
import numpy as np
import pytest

import asd_lattice as LT
from oracle import fft_oracle as F
from oracle import oracle as O


@pytest.mark.parametrize("L,pbc", [((5, 4, 3), (0, 0, 0)), ((4, 4, 4), (1, 1, 1)), ((6, 3, 4), (1, 1, 0))])
def test_sc_csr_matches_builders(L, pbc):
    xadj, adj, val = F.sc_csr(L, 1e-21, 1.5, pbc)
    bx, ba, bv = LT.build_csr(L, pbc, [1.5], [0] * 6, [0] * 6, LT.SC_NN, [LT._iso(1e-21)] * 6)
    assert np.array_equal(xadj, bx) and np.array_equal(adj, ba) and np.array_equal(val, bv)
    try:
        rx, ra, rv = O.ref_exchunitcell(L, pbc, [1.5], [(0, 0, v, np.eye(3) * 1e-21) for v in F.SC_NN],
                                        offdiag=False)
    except (OSError, AssertionError):
        pytest.skip("reference builders not built")
    assert np.array_equal(xadj, rx) and np.array_equal(adj, ra)
    assert np.array_equal(val[:, [0, 4, 8]], rv[:, [0, 4, 8]])


def test_dipole_nr_matches_library_builder():
    nr, mesh = F.dipole_nr((4, 3, 5))
    nr2, mesh2 = LT.dipole_nr((4, 3, 5))
    assert list(mesh) == list(mesh2)
    assert np.array_equal(nr, nr2)


def _small_system(L, update_pbc=(0, 0, 0)):
    return F.sc_dipole_system(L, pbc=update_pbc)


@pytest.mark.parametrize("L,update", [((6, 5, 4), 1), ((4, 4, 8), 3), ((3, 7, 2), 1)])
def test_fft_restatement_matches_direct_sum_oracle(L, update):
    s = _small_system(L)
    S0 = F.random_spins(s.nspins, 3)
    o = O.Oracle(s, dt=1e-16, update=update)
    o.set_spins(S0)
    f = F.FFTOracle(s, dt=1e-16, update=update, workers=2)
    f.set_spins(S0)
    # the field of the initial spins: exchange + long-range
    hf = f.field()
    ho = o.field()
    assert np.abs(hf - ho).max() <= 1e-12 * np.abs(ho).max()
    o.step(40)
    f.step(40)
    assert np.abs(f.spins() - o.spins()).max() <= 1e-12


def test_fft_restatement_exchange_in_nk():
    """ASD_LR_FFT: the whole field of every stage from N_k (exchange folded in)."""
    s = LT.sc_fft((4, 5, 3))
    S0 = F.random_spins(s.nspins, 5)
    o = O.Oracle(s, dt=1e-16)
    o.set_spins(S0)
    f = F.FFTOracle(s, dt=1e-16, workers=2)
    f.set_spins(S0)
    o.step(30)
    f.step(30)
    assert np.abs(f.spins() - o.spins()).max() <= 1e-12


def test_fft_restatement_refuses_finite_temperature():
    s = _small_system((3, 3, 3))
    s.temperature = 10.0
    with pytest.raises(NotImplementedError):
        F.FFTOracle(s)
