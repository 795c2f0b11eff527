"""Parity of the long-range field's plane kernels (z+y forward, x + N_k product + inverse x,
inverse y+z) with the FP64 oracle: the direct-sum oracle on small lattices, the FFT restatement
(itself pinned against the direct sum) on the sc 128x128x64 dipole lattice, and the cuFFT (x, y) passes
the plane kernels replace.

Tolerances: FP32 form max|dS| <= 1e-5 (and <= 1e-6 against the cuFFT passes, the same
arithmetic but for the transform's rounding); fused FP64 form with the FP32 long-range field
<= 1e-8 (the dipole field is ~1e-3 of the exchange field, its FP32 rounding enters at 1e-10 per
step); field read-back <= 1e-5 of the largest component."""
import numpy as np
import pytest

import asd_b200 as A
import asd_lattice as LT
from helpers import maxdiff
from oracle import fft_oracle as F
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def run(s, steps, precision, flags=0, update=1, S0=None):
    S0 = LT.random_spins(s.nspins, 0) if S0 is None else S0
    with A.Handle(A.RunParams(precision=precision, update=update, flags=flags), s) as h:
        h.set_spins(S0)
        h.step(steps)
        return h.get_spins(), h.tuning()


def oracle(s, steps, update=1, S0=None):
    S0 = LT.random_spins(s.nspins, 0) if S0 is None else S0
    o = O.Oracle(s, update=update)
    o.set_spins(S0)
    o.step(steps)
    return o.spins()


PLANES = "long-range: plane kernels"
CUFFT2D = "long-range: z-pass + cuFFT 2D planes"

# power-of-two meshes 2L: x in 4..64, y in 8..64 (the ky tile is 8), z in 8..64; the (8, 4, 2)
# lattice (mesh z 4) is below the plane kernels' sizes and runs the cuFFT planes
CASES = [(4, 4, 4), (8, 4, 2), (2, 8, 16), (16, 8, 8), (4, 16, 4), (8, 8, 32)]


@pytest.mark.parametrize("L", CASES)
@pytest.mark.parametrize("update", [1, 3])
def test_planes_dipole_csr(gpu, L, update):
    s = LT.sc_ferromagnet(L, pbc=(0, 0, 0), dipole=True)
    o = oracle(s, 40, update)
    g, tune = run(s, 40, A.FP32, A.FLAG_COMPENSATED, update)
    assert (CUFFT2D if L[2] < 4 else PLANES) in tune, tune
    assert maxdiff(g, o) <= 1e-5, maxdiff(g, o)
    c, _ = run(s, 40, A.FP32, A.FLAG_COMPENSATED | A.FLAG_CUFFT_PLANES, update)
    assert maxdiff(g, c) <= 1e-6, maxdiff(g, c)
    d, _ = run(s, 40, A.FP64_FUSED, 0, update)
    assert maxdiff(d, o) <= 1e-8, maxdiff(d, o)


@pytest.mark.parametrize("L,dims,off,path", [((3, 4, 2), (4, 4, 4), (1, 3, 2), PLANES),
                                             ((3, 4, 3), (4, 4, 4), (5, 4, 5), PLANES),
                                             ((5, 6, 3), (4, 8, 4), (1, 3, 2), CUFFT2D)])
def test_planes_box_away_from_origin(gpu, L, dims, off, path):
    """Spins in a box that starts at `off` of the mesh: the passes shift it to the origin.  A box
    wider than half the mesh runs the cuFFT planes."""
    s = LT.sc_ferromagnet(L, pbc=(0, 0, 0), dipole=True)
    nr, mesh = LT.dipole_nr(dims)
    s.mesh, s.nr = mesh, nr
    s.mesh_xyz = (LT.sc_mesh_xyz(L) + np.array(off, dtype=np.uint32)).astype(np.uint32)
    o = oracle(s, 30)
    g, tune = run(s, 30, A.FP32, A.FLAG_COMPENSATED)
    assert path in tune, tune
    assert maxdiff(g, o) <= 1e-5, maxdiff(g, o)
    d, _ = run(s, 30, A.FP64_FUSED)
    assert maxdiff(d, o) <= 1e-8, maxdiff(d, o)


def test_planes_general_interaction_matrix(gpu):
    """An interaction matrix that is neither symmetric nor even: 9 complex N_k components."""
    L = (4, 4, 4)
    s = LT.sc_ferromagnet(L, pbc=(0, 0, 0), dipole=True)
    rng = np.random.default_rng(7)
    s.nr = s.nr + rng.uniform(-0.05, 0.05, s.nr.shape) * np.abs(s.nr).max()
    o = oracle(s, 30)
    g, tune = run(s, 30, A.FP32, A.FLAG_COMPENSATED)
    assert PLANES in tune, tune
    assert maxdiff(g, o) <= 1e-5, maxdiff(g, o)
    c, _ = run(s, 30, A.FP32, A.FLAG_COMPENSATED | A.FLAG_CUFFT_PLANES)
    assert maxdiff(g, c) <= 1e-6, maxdiff(g, c)


@pytest.mark.parametrize("L", [(4, 4, 4), (8, 4, 8)])
def test_planes_fft_exchange_mode(gpu, L):
    """ASD_LR_FFT: the whole field from N_k (dipole + exchange folded in) at every stage."""
    s = LT.sc_fft(L)
    o = oracle(s, 40)
    g, tune = run(s, 40, A.FP32, A.FLAG_COMPENSATED)
    assert PLANES in tune, tune
    assert maxdiff(g, o) <= 1e-5, maxdiff(g, o)


def test_planes_field_readback(gpu):
    """Exchange + long-range field read-back after one step.  In the dipole mode the long-range
    part is the one evaluated from the step's initial spins (refreshed every `update` steps);
    the oracle evaluates it from the current spins, which differ by one step (a relative change of
    the field far below the tolerance)."""
    s = LT.sc_ferromagnet((8, 8, 4), pbc=(0, 0, 0), dipole=True)
    S0 = LT.random_spins(s.nspins, 2)
    o = O.Oracle(s)
    o.set_spins(S0)
    o.step(1)
    ho = o.field()
    for prec in (A.FP32, A.FP64_FUSED):
        with A.Handle(A.RunParams(precision=prec, flags=A.FLAG_COMPENSATED if prec == A.FP32 else 0), s) as h:
            h.set_spins(S0)
            h.step(1)
            hg = h.get_field()
        assert maxdiff(hg, ho) <= 1e-5 * np.abs(ho).max(), (prec, maxdiff(hg, ho))


def test_planes_sc128x128x64_lattice_against_fft_restatement(gpu):
    """The 1M-spin dipole lattice (sc 128x128x64, mesh 256x256x128), 10 steps, against the FFT
    restatement of the step on the host."""
    s = LT.sc_ferromagnet((128, 128, 64), pbc=(0, 0, 0), dipole=True)
    S0 = LT.random_spins(s.nspins, 0)
    f = F.FFTOracle(F.sc_dipole_system((128, 128, 64)), update=1)
    f.set_spins(S0)
    f.step(10)
    ref = f.spins()
    g, tune = run(s, 10, A.FP32, A.FLAG_COMPENSATED, S0=S0)
    assert PLANES in tune, tune
    assert maxdiff(g, ref) <= 1e-5, maxdiff(g, ref)
    d, _ = run(s, 10, A.FP64_FUSED, S0=S0)
    assert maxdiff(d, ref) <= 1e-8, maxdiff(d, ref)
    p, _ = run(s, 10, A.FP64_PLAIN, S0=S0)
    assert maxdiff(p, ref) <= 1e-10, maxdiff(p, ref)


def test_planes_shared_memory_limit_per_kernel(gpu):
    """Two x-pass kernels of one signature in one process, the larger first: a general N_k on
    mesh x 256 (191 KB of shared memory per block), then on mesh x 128 (96 KB).  Each kernel
    gets its own raised shared-memory limit, whatever the order of the handles."""
    rng = np.random.default_rng(7)
    for L in ((128, 4, 4), (64, 4, 4)):
        s = LT.sc_ferromagnet(L, pbc=(0, 0, 0), dipole=True)
        s.nr = s.nr + rng.uniform(-0.05, 0.05, s.nr.shape) * np.abs(s.nr).max()
        o = oracle(s, 10)
        g, tune = run(s, 10, A.FP32, A.FLAG_COMPENSATED)
        assert PLANES in tune, tune
        assert maxdiff(g, o) <= 1e-5, (L, maxdiff(g, o))


@pytest.mark.parametrize("update", [1, 2])
def test_planes_dipole_finite_temperature(gpu, update):
    """The plane-kernel dipole field at T = 300 K against the direct-sum oracle drawing the same
    Philox noise: the thermal field and the held long-range field together, with the dipole
    refreshed every step and every second step."""
    s = LT.sc_ferromagnet((8, 8, 4), pbc=(0, 0, 0), dipole=True, T=300.0)
    S0 = LT.random_spins(s.nspins, 3)
    o = O.Oracle(s, update=update, seed=7)
    o.set_spins(S0)
    o.step(40)
    ref = o.spins()
    for prec, flags, tol in ((A.FP32, A.FLAG_COMPENSATED, 1e-5), (A.FP64_FUSED, 0, 1e-8)):
        with A.Handle(A.RunParams(precision=prec, flags=flags, update=update, seed=7), s) as h:
            h.set_spins(S0)
            h.step(40)
            assert PLANES in h.tuning(), h.tuning()
            err = maxdiff(h.get_spins(), ref)
        assert err <= tol, (prec, err)
