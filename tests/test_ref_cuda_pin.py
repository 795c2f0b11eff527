"""The product against the reference's OWN CUDA step kernels, compiled from the reference sources
(src/cuint.cu, src/cufields.cu, src/cuintRK4.cu, src/cuintRK5.cu) and launched in the reference
driver's order (src/cuda.cu:43-258, src/cudaRK4.cu:38-233, src/cudaRK5.cu) by
oracle/ref_cuda_harness.cu, on the same GPU and the same inputs.

Tolerances: the reference kernels are built with nvcc's default FMA contraction and its double
rsqrt, the FP64 plain form without contraction and with IEEE 1/sqrt, so the two differ by a few
ulp per step: max|dS| <= 1e-10 over the runs below (T = 0).  At T > 0 the reference reads float
normals (Crand) where the FP64 forms use the double normals they were rounded from, so the bound
there is 1e-7.  The FP32 form is held to its usual 1e-5.
"""
import os

import numpy as np
import pytest

import asd_b200 as A
import asd_lattice as LT
from helpers import maxdiff, plaquette_quartets
from oracle import oracle as O

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(O.REF_CUDA_SO),
                                 reason="oracle/_ref/libref_cuda.so not built (needs the reference tree)")]


def run_both(s, steps, precision=A.FP64_PLAIN, integrator=A.HEUN, flags=0, dt=1e-16, applied=(0, 0, 0),
             anis=None, dzz=False, four_spin=None, noise=False, seed=1):
    S0 = LT.random_spins(s.nspins, 0)
    ref = O.RefCUDA(s, dt=dt, applied=applied, integrator=integrator, dzz_from_dyy=dzz, anis=anis)
    if four_spin is not None:
        ref.set_four_spin(*four_spin)
    ref.set_spins(S0)
    if noise:
        for t in range(steps):
            ref.set_noise(A.thermal_normals(seed, s.stream, t, s.nspins).astype(np.float32))
            ref.step(1)
    else:
        ref.step(steps)
    rs, rdet = ref.spins(), ref.det_field()
    ref.close()
    kw = dict(anis or {})
    p = A.RunParams(integrator=integrator, precision=precision, dt=dt, applied=applied, seed=seed,
                    flags=flags | (A.FLAG_COMPENSATED if precision == A.FP32 else 0), **kw)
    with A.Handle(p, s) as h:
        if four_spin is not None:
            h.set_four_spin(*four_spin[:4], four_spin[4], divide_by_3=True)
        h.set_spins(S0)
        h.step(steps)
        return h.get_spins(), h.get_det_field(), rs, rdet


@pytest.mark.parametrize("precision,tol", [(A.FP64_PLAIN, 1e-10), (A.FP64_FUSED, 1e-10), (A.FP32, 1e-5)])
def test_heun_csr_diagonal(gpu, precision, tol):
    s = LT.sc_ferromagnet(8)
    g, gdet, r, rdet = run_both(s, 300, precision)
    assert maxdiff(g, r) <= tol
    if precision == A.FP64_PLAIN:
        assert maxdiff(gdet, rdet) <= 1e-10 * np.abs(rdet).max()


@pytest.mark.parametrize("layout", ["csr", "dia"])
@pytest.mark.parametrize("dzz", [False, True])
def test_heun_full_tensor(gpu, layout, dzz):
    """BCT-2 full 3x3 tensors through CSpMV_CSR_OffDiag / CSpMV_DIA_OffDiag; with dzz the reference
    upload of Cdzz from datayy (src/cuda_util.cu:308-312) against FLAG_GPU_DZZ_FROM_DYY."""
    s = LT.bct2_antiferromagnet(3, layout=layout)
    flags = A.FLAG_GPU_DZZ_FROM_DYY if dzz else 0
    g, _, r, _ = run_both(s, 100, A.FP64_PLAIN, flags=flags, dzz=dzz)
    assert maxdiff(g, r) <= 1e-10
    g32, _, _, _ = run_both(s, 100, A.FP32, flags=flags, dzz=dzz)
    assert maxdiff(g32, r) <= 1e-5


def test_heun_dia_open_boundaries_site_field_and_anisotropy(gpu):
    """CSpMV_DIA with open z (col out of range skipped), the per-site field CHstg, the applied
    field and all four global anisotropy terms (src/cuint.cu:72-130)."""
    s = LT.sc_ferromagnet(6, exch="dia", pbc=(1, 0, 1))
    rng = np.random.default_rng(5)
    s.site_field = rng.normal(0.0, 2.0, (s.nspins, 3))
    k4p = np.eye(3).reshape(-1)
    k4q = np.array([[1, 1, 0], [1, -1, 0], [0, 0, 1]], dtype=float) / np.array([[2 ** .5], [2 ** .5], [1.0]])
    anis = dict(k2perp=2e-24, k2perpdir=(0.0, 0.6, 0.8), k2par=-1e-24, k2pardir=(1.0, 0.0, 0.0),
                k4perp=5e-25, k4perpdirs=tuple(k4p), k4par=-3e-25, k4pardirs=tuple(k4q.reshape(-1)))
    g, _, r, _ = run_both(s, 200, A.FP64_PLAIN, applied=(0.1, -0.2, 0.5), anis=anis)
    assert maxdiff(g, r) <= 1e-10
    g32, _, _, _ = run_both(s, 200, A.FP32, applied=(0.1, -0.2, 0.5), anis=anis)
    assert maxdiff(g32, r) <= 1e-5


def test_heun_four_spin(gpu):
    """CSpMV_CSR_FourSpin (src/cufields.cu:59-90, the division by 3 included)."""
    L = 5
    s = LT.sc_ferromagnet(L)
    q = plaquette_quartets(L)
    g, _, r, _ = run_both(s, 60, A.FP64_PLAIN, four_spin=(*q, 30.0))
    assert maxdiff(g, r) <= 1e-10


@pytest.mark.parametrize("integ", [A.RK4, A.RK5])
def test_rk_kernels(gpu, integ):
    """CdetRK4k1-4 + CdetSnp1 and CdetRK5k1-6 + CdetSnp1: the kernels carry the doubled rdt and the
    mixed stage spin, so the product runs with both RK flags."""
    s = LT.sc_ferromagnet(6, J2=-2e-22, exch="dia", pbc=(1, 1, 0))
    flags = A.FLAG_RK_DOUBLE_RDT | A.FLAG_RK_STAGE_SPIN_MIXED
    g, _, r, _ = run_both(s, 80, A.FP64_PLAIN, integrator=integ, flags=flags, dt=5e-16)
    assert maxdiff(g, r) <= 1e-10
    g0, _, _, _ = run_both(s, 80, A.FP64_PLAIN, integrator=integ, flags=0, dt=5e-16)
    assert maxdiff(g0, r) > 1e-8          # without the flags the dynamics differ


def test_heun_finite_temperature_same_normals(gpu):
    """T = 300 K: the reference reads the product's Philox normals rounded to float (Crand)."""
    s = LT.sc_ferromagnet(6, T=300.0)
    g, _, r, _ = run_both(s, 40, A.FP64_PLAIN, noise=True)
    d = maxdiff(g, r)
    assert d <= 1e-7, d
    g32, _, _, _ = run_both(s, 40, A.FP32, noise=True)
    assert maxdiff(g32, r) <= 1e-5


@pytest.mark.skipif(not os.path.exists(O.REF_SHIM_SO), reason="oracle/_ref/libref_shim.so not built")
@pytest.mark.parametrize("T", [0.0, 300.0])
def test_reference_side_binding(gpu, T):
    """The library behind the reference's own data contract: the namespace globals filled as the
    reference fills them, cullg::cuinit + cullg::llgGPU of gpu-atomistic-code_b200/shim/cullg_asd.cpp
    as llg::integrate calls them.  Equal bit for bit to the same run through asd_b200 directly,
    and (T = 0) to the reference's own kernels within the FP64 bound."""
    s = LT.sc_ferromagnet(6, T=T)
    S0 = LT.random_spins(s.nspins, 0)
    shim = O.RefShim(s, precision=A.FP64_PLAIN, seed=3)
    shim.set_spins(S0)
    S0n = shim.spins()          # as spins::Sx/Sy/Sz hold them: divided by their length once already
    shim.step(50)
    got = shim.spins()
    shim.close()
    assert maxdiff(got, S0) > 1e-3                 # the mirror was refreshed by real steps
    with A.Handle(A.RunParams(precision=A.FP64_PLAIN, seed=3), s) as h:
        h.set_spins(S0n)
        h.step(50)
        assert np.array_equal(got, h.get_spins())
    if T == 0.0:
        ref = O.RefCUDA(s)
        ref.set_spins(S0)
        ref.step(50)
        assert maxdiff(got, ref.spins()) <= 1e-10
        ref.close()


@pytest.mark.parametrize("name,builder", [
    ("bct2_64", lambda: LT.bct2_antiferromagnet(64, layout="csr", T=300.0)),
    ("bct2_64_dia", lambda: LT.bct2_antiferromagnet(64, layout="dia", T=300.0)),
    ("sc16", lambda: LT.sc_ferromagnet(16, T=300.0)),
])
def test_reference_kernels_timed(gpu, name, builder):
    """The reference's own Heun step on this GPU (cuRAND XORWOW draw, SpMV, CHeun1, SpMV, CHeun2 at
    256 threads per block, src/cuda.cu:43-258), timed like the library: untimed 256 MB write before
    each step, CUDA events per step.  Prints one JSON line per workload beside the library's FP32
    form on the same lattice; checks only that both ran and kept unit spins."""
    import json
    s = builder()
    S0 = LT.random_spins(s.nspins, 0)
    ref = O.RefCUDA(s, block=256)
    ref.enable_curand(1)
    ref.set_spins(S0)
    ref.step(3)
    steps = 20
    ms_ref = ref.time_steps_cold(steps)
    rs = ref.spins()
    ref.close()
    assert np.allclose(np.linalg.norm(rs, axis=1), 1.0, atol=1e-12)
    p = A.RunParams(precision=A.FP32, flags=A.FLAG_COMPENSATED | A.FLAG_AUTOTUNE, seed=1)
    with A.Handle(p, s) as h:
        h.set_spins(S0)
        h.step(3)
        ms_ours, _ = h.time_steps_cold(steps)
        assert np.allclose(np.linalg.norm(h.get_spins(), axis=1), 1.0, atol=1e-6)
    line = {"workload": name, "nspins": s.nspins, "steps": steps,
            "reference_cuda_fp64_spin_updates_per_s": s.nspins * steps / (ms_ref * 1e-3),
            "library_fp32_spin_updates_per_s": s.nspins * steps / (ms_ours * 1e-3)}
    print("REFTIMING " + json.dumps(line))
