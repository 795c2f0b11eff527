"""Parity of the CUDA path (through the C ABI) with the FP64 oracle on the same seeded inputs.

Tolerances:
  FP64 plain form: bit-exact (identical operation order, no FMA contraction, same noise);
  fused FP64 form: max|dS| <= 1e-10;
  FP32 form:       max|dS| <= 1e-5 (the accuracy bound for the FP32 state vs FP64);
  FFT paths (cuFFT rounding): FP64 <= 1e-10, FP32 <= 1e-5.
"""
import numpy as np
import pytest

import asd_b200 as A
import asd_lattice as LT
from helpers import maxdiff, plaquette_quartets
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def pair(systems, steps, precision, integrator=A.HEUN, flags=0, dt=1e-16, seed=1, update=1, applied=(0, 0, 0),
         spins=None, oracle_flags=None):
    if not isinstance(systems, list):
        systems = [systems]
    n = sum(s.nspins for s in systems)
    S0 = LT.random_spins(n, 0) if spins is None else spins
    p = A.RunParams(integrator=integrator, precision=precision, dt=dt, seed=seed, update=update, flags=flags,
                    applied=applied)
    with A.Handle(p, systems) as h:
        h.set_spins(S0)
        h.step(steps)
        g = h.get_spins()
        det = h.get_det_field()
    o = O.Oracle(systems, integrator=integrator, dt=dt, seed=seed, update=update, applied=applied,
                 flags=(flags & 0xFFFF) if oracle_flags is None else oracle_flags)
    o.set_spins(S0)
    o.step(steps)
    return g, o.spins(), det, o.det_field()


def test_thermal_normals_bit_exact(gpu):
    for seed, stream, step in [(1, 0, 0), (12345678901, 7, 2**33 + 5), (0, 95, 19999)]:
        g = A.thermal_normals(seed, stream, step, 3000)
        o = O.thermal_normals(seed, stream, 3000, step)
        assert np.array_equal(g, o)


def test_thermal_normals_f32_bit_exact(gpu):
    for seed, stream, step in [(1, 0, 0), (987654321, 3, 2**40 + 1)]:
        g = A.thermal_normals_f32(seed, stream, step, 2000)
        o = O.thermal_normals_f(seed, stream, 2000, step)
        assert np.array_equal(g, o)
        d = O.thermal_normals(seed, stream, 2000, step)
        assert np.abs(g - d).max() < 1e-5   # same Philox draw, float series


@pytest.mark.parametrize("T", [0.0, 300.0])
def test_plain_heun_csr_bit_exact(gpu, T):
    s = LT.sc_ferromagnet(8, T=T)
    g, o, dg, do = pair(s, 200, A.FP64_PLAIN)
    assert np.array_equal(g, o), maxdiff(g, o)
    assert np.array_equal(dg, do), maxdiff(dg, do)


def test_plain_full_tensor_csr_and_dia_bit_exact(gpu):
    s = LT.bct2_antiferromagnet(3, T=100.0)
    g, o, _, _ = pair(s, 60, A.FP64_PLAIN)
    assert np.array_equal(g, o), maxdiff(g, o)
    s = LT.bct2_antiferromagnet(3, layout="dia", T=100.0)
    g2, o2, _, _ = pair(s, 60, A.FP64_PLAIN)
    assert np.array_equal(g2, o2), maxdiff(g2, o2)
    s = LT.sc_ferromagnet(6, exch="dia", pbc=(1, 0, 1))
    g3, o3, _, _ = pair(s, 100, A.FP64_PLAIN)
    assert np.array_equal(g3, o3), maxdiff(g3, o3)


def test_plain_gpu_quirk_flags_bit_exact(gpu):
    s = LT.bct2_antiferromagnet(3)
    g, o, _, _ = pair(s, 40, A.FP64_PLAIN, flags=A.FLAG_GPU_DZZ_FROM_DYY)
    assert np.array_equal(g, o), maxdiff(g, o)
    g0, _, _, _ = pair(s, 40, A.FP64_PLAIN)
    assert maxdiff(g, g0) > 1e-8      # the Cdzz<-datayy upload bug changes the dynamics


@pytest.mark.parametrize("integ", [A.RK4, A.RK5])
@pytest.mark.parametrize("flags", [0, A.FLAG_RK_DOUBLE_RDT | A.FLAG_RK_STAGE_SPIN_MIXED])
def test_plain_rk_bit_exact(gpu, integ, flags):
    s = LT.sc_ferromagnet(6, J2=-2e-22, exch="dia", pbc=(1, 1, 0), T=50.0)
    g, o, _, _ = pair(s, 50, A.FP64_PLAIN, integrator=integ, flags=flags, dt=5e-16)
    assert np.array_equal(g, o), maxdiff(g, o)


LAYOUTS = [0, A.FLAG_STREAMED_EXCHANGE]   # typed (column, tensor id) and streamed tensors


@pytest.mark.parametrize("layout", LAYOUTS)
def test_fused_fp64_close(gpu, layout):
    s = LT.sc_ferromagnet(8, T=0.0)
    g, o, _, _ = pair(s, 300, A.FP64_FUSED, flags=layout)
    assert maxdiff(g, o) <= 1e-10
    s = LT.bct2_antiferromagnet(3, T=0.0)
    g, o, _, _ = pair(s, 100, A.FP64_FUSED, flags=layout)
    assert maxdiff(g, o) <= 1e-10
    s = LT.bct2_antiferromagnet(3, layout="dia", T=0.0)
    g, o, _, _ = pair(s, 100, A.FP64_FUSED, flags=layout)
    assert maxdiff(g, o) <= 1e-10


@pytest.mark.parametrize("flags", [0, A.FLAG_COMPENSATED, A.FLAG_COMPENSATED | A.FLAG_STREAMED_EXCHANGE])
def test_fp32_sc_close(gpu, flags):
    s = LT.sc_ferromagnet(10, T=0.0)
    g, o, _, _ = pair(s, 1000, A.FP32, flags=flags)
    assert maxdiff(g, o) <= 1e-5, maxdiff(g, o)


@pytest.mark.parametrize("layout", LAYOUTS)
def test_fp32_bct_full_csr_and_dia_close(gpu, layout):
    for kind in ("csr", "dia"):
        s = LT.bct2_antiferromagnet(4, layout=kind, T=0.0)
        g, o, _, _ = pair(s, 300, A.FP32, flags=A.FLAG_COMPENSATED | layout)
        assert maxdiff(g, o) <= 1e-5, (kind, maxdiff(g, o))


def test_fp32_many_distinct_tensors_fall_back_to_streamed(gpu):
    s = LT.sc_ferromagnet(7, T=0.0)
    rng = np.random.default_rng(8)
    s.csr_val = s.csr_val * rng.uniform(0.5, 1.5, size=(len(s.adjncy), 1))   # > 256 distinct tensors
    for prec, tol in ((A.FP32, 1e-5), (A.FP64_FUSED, 1e-10)):
        g, o, _, _ = pair(s, 200, prec, flags=A.FLAG_COMPENSATED)
        assert maxdiff(g, o) <= tol


@pytest.mark.parametrize("integ", [A.RK4, A.RK5])
@pytest.mark.parametrize("layout", LAYOUTS)
def test_fp32_rk_close(gpu, integ, layout):
    s = LT.sc_ferromagnet(8, J2=-2e-22, exch="dia", pbc=(1, 1, 0), T=0.0)
    g, o, _, _ = pair(s, 200, A.FP32, integrator=integ, dt=5e-16, flags=A.FLAG_COMPENSATED | layout)
    assert maxdiff(g, o) <= 1e-5, maxdiff(g, o)


def test_fp32_finite_temperature_close(gpu):
    """FP32 noise is the float series on the same Philox draw: the trajectory stays within 1e-5."""
    s = LT.sc_ferromagnet(8, T=300.0)
    g, o, _, _ = pair(s, 100, A.FP32, flags=A.FLAG_COMPENSATED)
    assert maxdiff(g, o) <= 1e-5, maxdiff(g, o)


# mesh 2L per axis: L = 6 takes the full 3D transform (last axis 12); the others the pruned one
# with N = m_z/2 = 4, 8 (odd box extents in x and y), 64, 128, 256 (two register passes) and 512
# (radix-2 passes in shared memory)
@pytest.mark.parametrize("L", [6, (8, 6, 4), (5, 7, 8), (6, 5, 64), (4, 3, 128), (2, 2, 256), (2, 2, 512)])
def test_dipole_csr_plain_and_fp32(gpu, L):
    s = LT.sc_ferromagnet(L, pbc=(0, 0, 0), dipole=True)
    g, o, _, _ = pair(s, 40, A.FP64_PLAIN, update=1)
    assert maxdiff(g, o) <= 1e-10, maxdiff(g, o)
    g, o, _, _ = pair(s, 40, A.FP32, update=1, flags=A.FLAG_COMPENSATED)
    assert maxdiff(g, o) <= 1e-5, maxdiff(g, o)
    g, o, _, _ = pair(s, 40, A.FP32, update=5, flags=A.FLAG_COMPENSATED)
    assert maxdiff(g, o) <= 1e-5, maxdiff(g, o)


@pytest.mark.parametrize("L", [6, (8, 6, 4), (5, 7, 8)])
def test_fft_exchange_mode_plain_and_fp32(gpu, L):
    s = LT.sc_fft(L)
    g, o, _, _ = pair(s, 40, A.FP64_PLAIN)
    assert maxdiff(g, o) <= 1e-10, maxdiff(g, o)
    g, o, _, _ = pair(s, 40, A.FP32, flags=A.FLAG_COMPENSATED)
    assert maxdiff(g, o) <= 1e-5, maxdiff(g, o)


def test_field_readback_matches_oracle(gpu):
    s = LT.bct2_antiferromagnet(3)
    S0 = LT.random_spins(s.nspins, 4)
    o = O.Oracle(s)
    o.set_spins(S0)
    ho = o.field()
    for prec, tol, fl in [(A.FP64_PLAIN, 0.0, 0), (A.FP64_FUSED, 1e-12, 0), (A.FP32, 1e-5, 0),
                          (A.FP32, 1e-5, A.FLAG_STREAMED_EXCHANGE)]:
        with A.Handle(A.RunParams(precision=prec, flags=fl), s) as h:
            h.set_spins(S0)
            hg = h.get_field()
        assert maxdiff(hg, ho) <= tol * np.abs(ho).max(), (prec, maxdiff(hg, ho))


def test_replicas_batched_equal_individual(gpu):
    reps = [LT.sc_ferromagnet(4, T=10.0, stream=0), LT.sc_ferromagnet(5, T=200.0, stream=1),
            LT.sc_ferromagnet(3, T=0.0, stream=2)]
    for prec in (A.FP64_PLAIN, A.FP32):
        S = [LT.random_spins(r.nspins, 10 + k) for k, r in enumerate(reps)]
        p = A.RunParams(precision=prec, seed=9)
        with A.Handle(p, reps) as h:
            h.set_spins(np.concatenate(S))
            h.step(70)
            gb = h.get_spins()
            m = h.magnetisation()
        off = 0
        for k, r in enumerate(reps):
            with A.Handle(p, r) as h1:
                h1.set_spins(S[k])
                h1.step(70)
                g1 = h1.get_spins()
            assert np.array_equal(gb[off:off + r.nspins], g1)
            assert np.allclose(m[k, 0], g1.mean(axis=0), rtol=0, atol=1e-14)
            off += r.nspins
    o = O.Oracle(reps, seed=9)
    o.set_spins(np.concatenate(S))
    o.step(70)
    with A.Handle(A.RunParams(precision=A.FP64_PLAIN, seed=9), reps) as h:
        h.set_spins(np.concatenate(S))
        h.step(70)
        assert np.array_equal(h.get_spins(), o.spins())


def test_site_field_ramp_bit_exact(gpu):
    s = LT.sc_ferromagnet(5)
    prof = np.random.default_rng(3).normal(size=(s.nspins, 3)) * 5.0
    s.site_field = prof
    S0 = LT.random_spins(s.nspins, 1)
    o = O.Oracle(s)
    o.set_spins(S0)
    O.olib().orc_set_site_field(o.c, O._ptr(O.a64(prof), O.C.c_double), 0.25)
    o.step(30)
    with A.Handle(A.RunParams(precision=A.FP64_PLAIN), s) as h:
        h.set_spins(S0)
        h.set_site_field_scale(0.25)
        h.step(30)
        assert np.array_equal(h.get_spins(), o.spins())
    with A.Handle(A.RunParams(precision=A.FP32, flags=A.FLAG_COMPENSATED), s) as h:
        h.set_spins(S0)
        h.set_site_field_scale(0.25)
        h.step(30)
        assert maxdiff(h.get_spins(), o.spins()) <= 1e-5


def test_edge_cases(gpu):
    # one spin, no exchange
    s = A.SpinSystem(nspins=1, materials=[A.MaterialSpec()], exch=A.EXCH_NONE)
    g, o, _, _ = pair(s, 50, A.FP64_PLAIN, applied=(0, 0, 3.0), spins=np.array([[1.0, 0, 0]]))
    assert np.array_equal(g, o)
    # ragged rows (open boundaries), rows with no neighbours, N not a multiple of 32
    s = LT.sc_ferromagnet((3, 5, 7), pbc=(0, 0, 0))
    xadj = s.xadj.copy()
    adj = list(s.adjncy)
    val = list(s.csr_val)
    # isolate spin 0: drop its row entries and the entries pointing at it
    keep = []
    rows = []
    for i in range(s.nspins):
        r = [(j, v) for j, v in zip(adj[xadj[i]:xadj[i + 1]], val[xadj[i]:xadj[i + 1]]) if i != 0 and j != 0]
        rows.append(r)
    s.xadj = np.concatenate([[0], np.cumsum([len(r) for r in rows])]).astype(np.uint32)
    s.adjncy = np.array([j for r in rows for j, _ in r], dtype=np.uint32)
    s.csr_val = np.array([v for r in rows for _, v in r])
    for prec, tol in [(A.FP64_PLAIN, 0.0), (A.FP32, 1e-5)]:
        g, o, _, _ = pair(s, 100, prec)
        assert maxdiff(g, o) <= tol


def test_errors_are_reported_not_fatal(gpu):
    s = LT.sc_ferromagnet(4)
    with A.Handle(A.RunParams(precision=A.FP32), s) as h:
        bad = LT.random_spins(s.nspins, 0)
        bad[3, 1] = np.nan
        with pytest.raises(A.AsdError) as e:
            h.set_spins(bad)
        assert e.value.code == A.ASD_ENOTFINITE
        with pytest.raises(A.AsdError):
            h.set_spins(np.zeros((s.nspins, 3)))
        h.step(3)               # the handle is still usable
    s2 = LT.sc_ferromagnet(4)
    s2.adjncy = s2.adjncy.copy()
    s2.adjncy[5] = 10**6
    with pytest.raises(A.AsdError) as e:
        A.Handle(A.RunParams(), s2)
    assert e.value.code == A.ASD_EINVAL


def test_site_field_pulse(gpu):
    """Gaussian-in-time envelope on the site field (the config-4 pulse): plain form bit-exact."""
    s = LT.sc_ferromagnet(5)
    s.site_field = np.random.default_rng(5).normal(size=(s.nspins, 3)) * 20.0
    amp, t0, sig, dt = 0.8, 20e-16, 8e-16, 1e-16
    S0 = LT.random_spins(s.nspins, 2)
    o = O.Oracle(s, dt=dt)
    o.set_site_scale(0.5)
    o.set_pulse(amp, t0, sig, dt)
    o.set_spins(S0)
    o.step(40)
    for prec, tol in ((A.FP64_PLAIN, 0.0), (A.FP32, 1e-5)):
        with A.Handle(A.RunParams(precision=prec, dt=dt, flags=A.FLAG_COMPENSATED if prec == A.FP32 else 0), s) as h:
            h.set_spins(S0)
            h.set_site_field_scale(0.5)
            h.set_site_field_pulse(amp, t0, sig)
            h.step(40)
            assert maxdiff(h.get_spins(), o.spins()) <= tol, (prec, maxdiff(h.get_spins(), o.spins()))


def test_magnetisation_stats_running_welford(gpu):
    """Device RunningStat of |m_s| (sim::MvT) against a host Welford over the oracle trajectory."""
    reps = [LT.sc_ferromagnet(4, T=50.0, stream=0), LT.sc_ferromagnet(5, T=150.0, stream=1)]
    S = np.concatenate([LT.random_spins(r.nspins, 3 + k) for k, r in enumerate(reps)])
    o = O.Oracle(reps, seed=4)
    o.set_spins(S)
    n = np.zeros(2); mean = np.zeros(2); m2 = np.zeros(2); prev = np.zeros(2)
    with A.Handle(A.RunParams(precision=A.FP64_PLAIN, seed=4), reps) as h:
        h.set_spins(S)
        for k in range(25):
            h.step(2)
            h.sample_magnetisation()
            o.step(2)
            x = np.linalg.norm(o.magnetisation()[:, 0, :], axis=1)
            n += 1
            prev = mean.copy()
            d = x - mean
            mean = mean + d / n
            m2 = m2 + d * (x - mean)
        st = h.magnetisation_stats()[:, 0, :]
        assert np.array_equal(st[:, 0], n)
        assert np.allclose(st[:, 1], mean, rtol=1e-12, atol=0)
        assert np.allclose(st[:, 2], m2 / (n - 1), rtol=1e-9, atol=1e-18)
        assert np.allclose(st[:, 3], prev, rtol=1e-12, atol=0)
        h.reset_magnetisation_stats()
        assert np.all(h.magnetisation_stats() == 0)


@pytest.mark.parametrize("prec", [A.FP64_PLAIN, A.FP32, A.FP64_FUSED])
def test_sq_sampler_matches_fftn(gpu, prec):
    """S(q,t) series: psi_k of psi = uo_a S_a + i uo_b S_b on the mesh, forward transform (FFTW sign)."""
    rng = np.random.default_rng(11)
    cases = [(LT.sc_ferromagnet((6, 5, 4), T=200.0), (6, 5, 4), 2, None),
             (LT.bct2_antiferromagnet(3, T=50.0), (6, 3, 3), 0, np.array([[1.0, 1, 1], [-1, -1, 1]]))]
    for s, mesh, qaxis, uo in cases:
        n = s.nspins
        xyz = np.stack(np.unravel_index(rng.permutation(np.prod(mesh))[:n], mesh), axis=1).astype(np.uint32)
        kp = np.stack(np.unravel_index(rng.choice(np.prod(mesh), 9, replace=False), mesh), axis=1).astype(np.uint32)
        atom = np.arange(n) % len(s.materials) if s.atom is None else np.asarray(s.atom)
        sub = np.array([s.materials[m].sublattice for m in atom])
        u = np.ones((int(sub.max()) + 1, 3)) if uo is None else uo
        flags = A.FLAG_COMPENSATED if prec == A.FP32 else 0
        with A.Handle(A.RunParams(precision=prec, flags=flags), s) as h:
            h.set_spins(LT.random_spins(n, 4))
            h.sq_setup(mesh, xyz, kp, max_samples=4, qaxis=qaxis, uo=uo)
            want = []
            for _ in range(3):
                h.step(5)
                h.sq_sample()
                want.append(O.sq_psi_k(h.get_spins(), sub, u, mesh, xyz, kp, qaxis))
            got = h.sq_series()
            assert got.shape == (3, 9)
            tol = 1e-12 if prec != A.FP32 else 1e-5
            assert np.abs(got - np.array(want)).max() <= tol * np.sqrt(n)
            h.sq_sample()
            with pytest.raises(A.AsdError):
                h.sq_sample()      # series full


def test_dsf_peaks_fp32_match_fp64_oracle(gpu):
    """Spin-wave film (J1+J2 DIA, RK4, Gaussian-in-time x sinc-in-space pulse): the DSF computed on
    the device equals the time-series restatement applied to the device series, the FP64 plain
    series equals the oracle trajectory's, and the FP32 run finds the same peak bins."""
    # the sinc profile varies along x only, so the pulse excites the (k, 0, 0) magnons; the
    # peak bins rise with k (the dispersion) and are separated from their neighbours by far
    # more than the FP32 error
    s = LT.film_dia(16, 16, 2, dipole=False, pulse_width_sites=2.0)
    n, dt, every, ns = s.nspins, 5e-16, 20, 512
    mesh, xyz = (16, 16, 2), LT.sc_mesh_xyz((16, 16, 2))
    kp = np.array([[k, 0, 0] for k in range(1, 9)], dtype=np.uint32)
    sub = np.zeros(n, dtype=np.int64)
    uo = np.ones((1, 3))
    S0 = np.tile([0.0, 0.0, 1.0], (n, 1))
    amp, t0, sig = 0.1, 20 * dt, 5 * dt
    sdt = every * dt
    spec = dict(window=0, width_hz=1.0 / (ns * sdt), sample_dt=sdt, fcut_lo=1e12, fcut_hi=1e15)
    o = O.Oracle(s, integrator=A.RK4, dt=dt)
    o.set_pulse(amp, t0, sig, dt)
    o.set_spins(S0)
    want = []
    for _ in range(ns):
        o.step(every)
        want.append(O.sq_psi_k(o.spins(), sub, uo, mesh, xyz, kp))
    want = np.array(want)
    _, _, pr_o, ps_o = O.sq_spectrum(want, np.prod(mesh), **spec)
    for prec in (A.FP64_PLAIN, A.FP32):
        flags = A.FLAG_COMPENSATED if prec == A.FP32 else 0
        with A.Handle(A.RunParams(integrator=A.RK4, precision=prec, dt=dt, flags=flags), s) as h:
            h.set_spins(S0)
            h.set_site_field_pulse(amp, t0, sig)
            h.sq_setup(mesh, xyz, kp, max_samples=ns)
            for _ in range(ns):
                h.step(every)
                h.sq_sample()
            got = h.sq_series()
            raw, sm, pr, ps = h.sq_spectrum(**spec)
        r2, s2, pr2, ps2 = O.sq_spectrum(got, np.prod(mesh), **spec)
        np.testing.assert_allclose(raw, r2, rtol=1e-9, atol=1e-300)
        np.testing.assert_allclose(sm, s2, rtol=1e-9, atol=1e-300)
        assert np.array_equal(pr, pr2) and np.array_equal(ps, ps2)
        if prec == A.FP64_PLAIN:
            assert np.abs(got - want).max() <= 1e-9 * np.sqrt(n)
        assert np.array_equal(ps, ps_o), (prec, ps, ps_o)
        assert np.array_equal(pr, pr_o), (prec, pr, pr_o)
    assert np.all(np.diff(ps_o.astype(int)) >= 0) and ps_o[-1] > ps_o[0]


@pytest.mark.parametrize("prec", [A.FP32, A.FP64_FUSED])
def test_launch_shapes_and_staging_bit_identical(gpu, prec):
    """Every block size, with no staging, bulk staging of the typed SELL words, and staging of
    the words plus the neighbour spins, and the autotuner's choice give bit-identical spins
    (each thread's arithmetic does not depend on the shape); no staging wait runs out."""
    s = LT.bct2_antiferromagnet(6, T=300.0)
    S0 = LT.random_spins(s.nspins, 8)
    flags = A.FLAG_COMPENSATED if prec == A.FP32 else 0
    outs = []
    names = {0: "staging=direct", 1: "staging=words ", 2: "staging=words+spins"}
    for shape in [(256, 1), (256, 0), (256, 2), (128, 2), (128, 1), (64, 2), (64, 0), None]:
        f = flags | (A.FLAG_AUTOTUNE if shape is None else 0)
        with A.Handle(A.RunParams(precision=prec, flags=f, seed=3), s) as h:
            if shape is not None:
                h.set_launch_shape(*shape)
                assert names[shape[1]] in h.tuning() + " ", h.tuning()
            else:
                assert "ms per stage launch" in h.tuning(), h.tuning()
            h.set_spins(S0)
            h.step(70)
            h.sync()
            outs.append(h.get_spins())
    for o in outs[1:]:
        assert np.array_equal(o, outs[0])
    g, o, _, _ = pair(s, 70, prec, flags=flags, seed=3, spins=S0)
    assert np.array_equal(g, outs[0])
    assert maxdiff(g, o) <= (1e-5 if prec == A.FP32 else 1e-10)


@pytest.mark.parametrize("prec", [A.FP32, A.FP64_FUSED])
def test_dia_input_on_both_device_layouts_bit_identical(gpu, prec):
    """A DIA matrix runs either on the DIA gather or as SELL-32 with its entries in ascending
    diagonal order; the two device layouts give bit-identical spins and fields."""
    for s in (LT.bct2_antiferromagnet(4, layout="dia", T=200.0), LT.film_dia(12, 10, 3, dipole=False)):
        S0 = LT.random_spins(s.nspins, 6)
        flags = A.FLAG_COMPENSATED if prec == A.FP32 else 0
        out = []
        for lay in (A.EXCH_DIA, A.EXCH_CSR):
            with A.Handle(A.RunParams(precision=prec, flags=flags, seed=2, integrator=A.RK4), s) as h:
                h.set_device_layout(lay)
                h.set_spins(S0)
                h.step(30)
                out.append((h.get_spins(), h.get_field()))
        assert np.array_equal(out[0][0], out[1][0])
        assert np.array_equal(out[0][1], out[1][1])


TTM = dict(gamma_e=3.0e3, Cl=2.0e6, G_ep=1.0e17, pump_time=2e-15, pump_fluence=4e21, cooling_time=1e-12,
           initial_T=40.0, pulses=[(1.0, 3e-15), (0.5, 6e-15)])


@pytest.mark.parametrize("prec,tol", [(A.FP64_PLAIN, 1e-12), (A.FP32, 1e-5)])
def test_two_temperature_model_drives_the_bath(gpu, prec, tol):
    """The device two-temperature model (CalcTe, src/laser_heating.cpp:884-895) advances Te and Tl
    like the restatement, and the spins follow the oracle stepped at the same bath temperature."""
    s = LT.sc_ferromagnet(5, T=0.0)
    S0 = LT.random_spins(s.nspins, 3)
    dt, nsteps, start = 1e-16, 60, 7
    o = O.Oracle(s, dt=dt, seed=5)
    o.set_spins(S0)
    o.step(start)
    prm = dict(TTM, t0=start)
    st = [TTM["initial_T"], TTM["initial_T"]]
    flags = A.FLAG_COMPENSATED if prec == A.FP32 else 0
    with A.Handle(A.RunParams(precision=prec, dt=dt, seed=5, flags=flags), s) as h:
        h.set_spins(S0)
        h.step(start)
        h.set_ttm(**TTM)
        for k in range(nsteps):
            T = O.ttm_step(st, prm, start + k, dt)
            o.set_temperatures([T])
            o.step(1)
            h.step(1)
            if k % 10 == 9:
                te, tl = h.ttm_temperatures()
                assert abs(te - st[0]) <= 1e-12 * st[0] and abs(tl - st[1]) <= 1e-12 * st[1]
        assert st[0] > 2 * TTM["initial_T"]          # the pulses heated the electrons
        assert maxdiff(h.get_spins(), o.spins()) <= tol
        h.set_ttm(off=True)
        h.step(3)


@pytest.mark.parametrize("div3", [True, False])
def test_four_spin_term(gpu, div3):
    """Four-spin exchange (src/cufields.cu:59-90): the FP64 plain form equals the oracle bit for bit
    (with and without the GPU path's division by 3), the fused forms to their tolerances."""
    L = 5
    s = LT.sc_ferromagnet(L, T=100.0)
    q = plaquette_quartets(L)
    jq = 30.0                                   # [T], comparable to the exchange field
    S0 = LT.random_spins(s.nspins, 9)
    for prec, tol in ((A.FP64_PLAIN, 0.0), (A.FP64_FUSED, 1e-10), (A.FP32, 1e-5)):
        o = O.Oracle(s, seed=2)
        o.set_four_spin(*q, jq, div3)
        o.set_spins(S0)
        o.step(60)
        flags = A.FLAG_COMPENSATED if prec == A.FP32 else 0
        with A.Handle(A.RunParams(precision=prec, seed=2, flags=flags), s) as h:
            h.set_four_spin(*q, jq, divide_by_3=div3)
            h.set_spins(S0)
            h.step(60)
            d = maxdiff(h.get_spins(), o.spins())
            assert d <= tol, (prec, d)
            if prec == A.FP64_PLAIN:
                assert np.array_equal(h.get_field(), o.field())


@pytest.mark.parametrize("prec", [A.FP32, A.FP64_FUSED])
def test_dependent_launch_bit_identical(gpu, prec):
    """Programmatic dependent launch (the default: each step kernel's blocks may become resident
    while its predecessor finishes, and wait for it before touching memory) against strictly
    ordered launches (ASD_FLAG_SERIAL_LAUNCH), through the 32-step graphs, the one-step graph
    and direct launches: bit-identical spins at finite temperature, with the plane-kernel dipole
    field and with RK4."""
    cases = [(LT.bct2_antiferromagnet(5, T=300.0), {}),
             (LT.sc_ferromagnet((16, 16, 8), pbc=(0, 0, 0), dipole=True, T=100.0), {}),
             (LT.film_dia(12, 10, 3, dipole=True), dict(integrator=A.RK4))]
    for s, kw in cases:
        S0 = LT.random_spins(s.nspins, 12)
        base = A.FLAG_COMPENSATED if prec == A.FP32 else 0
        outs = []
        for flags, single in ((base, False), (base | A.FLAG_SERIAL_LAUNCH, False), (base, True)):
            with A.Handle(A.RunParams(precision=prec, flags=flags, seed=5, **kw), s) as h:
                h.set_spins(S0)
                if single:
                    for _ in range(70):
                        h.step(1)
                else:
                    h.step(70)                         # two 32-step graphs and 6 direct steps
                outs.append(h.get_spins())
        assert np.array_equal(outs[0], outs[1]), (s.nspins, maxdiff(outs[0], outs[1]))
        assert np.array_equal(outs[0], outs[2]), (s.nspins, maxdiff(outs[0], outs[2]))
