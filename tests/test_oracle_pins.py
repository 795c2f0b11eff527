"""The oracle pinned against the reference: golden vectors produced by the
reference's own llgCPU compiled from source (tests/golden/make_golden.py),
Philox known-answer vectors, and analytic single-spin dynamics."""
import math
import os
import subprocess

import numpy as np
import pytest

import asd_lattice as LT
from helpers import load, maxdiff, system_from_npz
from oracle import oracle as O

COMPAT = O.CPU_SUM_ORDER | O.CPU_CORRECTOR_ACCUM | O.CPU_THERMAL_Z_FROM_X


@pytest.mark.parametrize("name", ["ref_sc6_csr_T0_200.npz", "ref_bct3_csr_full_T0_100.npz", "ref_sc6_dia_T0_100.npz"])
def test_oracle_compat_reproduces_reference_llgcpu_T0(name):
    d = load(name)
    s = system_from_npz(d)
    o = O.Oracle(s, flags=COMPAT, noise=O.NOISE_MWC)
    o.set_spins(d["S0"])
    o.step(int(d["steps"]))
    assert np.array_equal(o.spins(), d["out"]), maxdiff(o.spins(), d["out"])


def test_oracle_compat_reproduces_reference_llgcpu_mwc_noise():
    d = load("ref_sc6_csr_T300_mwc_50.npz")
    s = system_from_npz(d)
    a, b = (int(x) for x in d["mwc"])
    o = O.Oracle(s, flags=COMPAT, noise=O.NOISE_MWC, mwc=(a, b))
    o.set_spins(d["S0"])
    o.step(int(d["steps"]))
    assert np.array_equal(o.spins(), d["out"]), maxdiff(o.spins(), d["out"])


def test_oracle_compat_reproduces_reference_llgcpu_recorded_noise():
    d = load("ref_sc4_open_T300_replay_20.npz")
    s = system_from_npz(d)
    o = O.Oracle(s, flags=COMPAT, noise=O.NOISE_BUFFER, noise_buf=d["noise"])
    o.set_spins(d["S0"])
    o.step(int(d["steps"]))
    assert np.array_equal(o.spins(), d["out"]), maxdiff(o.spins(), d["out"])


def test_oracle_compat_reproduces_reference_llgcpu_four_spin():
    """llgCPU's four-spin field H4s (no division by 3, recomputed at each stage) as a separate term."""
    d = load("ref_sc5_fourspin_T300_mwc_30.npz")
    s = system_from_npz(d)
    a, b = (int(x) for x in d["mwc"])
    o = O.Oracle(s, flags=COMPAT, noise=O.NOISE_MWC, mwc=(a, b))
    o.set_four_spin(d["q4_xadj"], d["q4_j"], d["q4_k"], d["q4_l"], float(d["q4_jq"]), False)
    o.set_spins(d["S0"])
    o.step(int(d["steps"]))
    assert np.array_equal(o.spins(), d["out"]), maxdiff(o.spins(), d["out"])


def test_recorded_noise_is_the_philox_stream():
    d = load("ref_sc4_open_T300_replay_20.npz")
    n = int(d["nspins"])
    xi = np.concatenate([O.thermal_normals(5, 0, n, t).reshape(-1) for t in range(int(d["steps"]))])
    assert np.array_equal(xi, d["noise"])


def test_clean_mode_differs_by_the_corrector_quirk():
    """The CPU corrector accumulates H(S)+H(S') (src/llgCPU.cpp:58-60,253-274): clean != compat."""
    d = load("ref_sc6_csr_T0_200.npz")
    s = system_from_npz(d)
    o = O.Oracle(s)
    o.set_spins(d["S0"])
    o.step(10)
    c = O.Oracle(s, flags=O.CPU_SUM_ORDER | O.CPU_CORRECTOR_ACCUM, noise=O.NOISE_MWC)
    c.set_spins(d["S0"])
    c.step(10)
    assert maxdiff(o.spins(), c.spins()) > 1e-4
    c2 = O.Oracle(s, flags=O.CPU_SUM_ORDER)
    c2.set_spins(d["S0"])
    c2.step(10)
    assert maxdiff(o.spins(), c2.spins()) < 1e-13   # only the summation order differs


def test_philox_known_answers():
    # Random123 known-answer vectors for philox4x32-10
    assert [int(x) for x in O.philox([0, 0, 0, 0], [0, 0])] == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert [int(x) for x in O.philox([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2)] == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert [int(x) for x in O.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0])] == \
        [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def test_series_log_and_sincos_accuracy():
    L = O.olib()
    for x in np.concatenate([np.geomspace(1e-300, 1, 200), np.linspace(0.01, 1, 200)]):
        assert abs(L.orc_log(float(x)) - math.log(x)) <= 4e-16 * max(1.0, abs(math.log(x)))
    import ctypes as C
    s, c = C.c_double(), C.c_double()
    for xv in list(range(0, 2**32, 2**32 // 997)) + [0, 2**32 - 1, 2**29, 2**30, 3 * 2**30]:
        L.orc_sincos_2pi(xv, C.byref(s), C.byref(c))
        ang = 2 * math.pi * (xv + 0.5) / 2**32
        assert abs(s.value - math.sin(ang)) < 1e-15 and abs(c.value - math.cos(ang)) < 1e-15


def test_normals_statistics():
    xi = O.thermal_normals(11, 3, 40000, 7).reshape(-1)
    assert abs(xi.mean()) < 0.01 and abs(xi.var() - 1.0) < 0.02
    # fourth moment of N(0,1) is 3
    assert abs((xi ** 4).mean() - 3.0) < 0.1


def test_single_spin_precession_matches_analytic():
    """One spin in a uniform field B z, lambda: S_z(t) = tanh(lambda*gamma*B*t/(1+lambda^2) + atanh(S_z(0)))."""
    import asd_b200 as A
    lam, B, dt = 0.1, 10.0, 1e-15
    s = A.SpinSystem(nspins=1, materials=[A.MaterialSpec(mu=2.0, lam=lam, k1u=0.0)])
    o = O.Oracle(s, dt=dt, applied=(0.0, 0.0, B))
    th = 1.0
    o.set_spins([[math.sin(th), 0.0, math.cos(th)]])
    nst = 2000
    o.step(nst)
    t = nst * dt
    sz = math.tanh(lam * A.GYRO * B * t / (1 + lam * lam) + math.atanh(math.cos(th)))
    assert abs(o.spins()[0, 2] - sz) < 2e-7      # Heun error at dt=1e-15
    phi = math.atan2(o.spins()[0, 1], o.spins()[0, 0])
    # precession about +z at gamma B/(1+lambda^2), counter-clockwise for llgpf=-1/(1+lambda^2)
    w = A.GYRO * B / (1 + lam * lam)
    expect = (w * t + math.pi) % (2 * math.pi) - math.pi
    assert abs(((phi - expect + math.pi) % (2 * math.pi)) - math.pi) < 1e-4


def test_oracle_applied_field_change_between_steps():
    """set_applied between steps (the reference's field ramp, src/ramp_field.cpp:221-223) gives
    the run of an oracle built with that field from the same spins and step on (to the rounding
    of set_spins' renormalisation), and one kept at the old field differs."""
    s = LT.sc_ferromagnet(4, T=30.0)
    S = LT.random_spins(s.nspins, 6)
    a = O.Oracle(s, applied=(0.0, 0.0, 0.5))
    a.set_spins(S)
    a.step(5)
    a.set_applied((0.3, -0.2, 1.0))
    mid = a.spins().copy()
    b = O.Oracle(s, applied=(0.3, -0.2, 1.0))
    b.set_spins(mid)
    b.t = a.t
    a.step(7)
    b.step(7)
    assert maxdiff(a.spins(), b.spins()) <= 1e-13, maxdiff(a.spins(), b.spins())
    c = O.Oracle(s, applied=(0.0, 0.0, 0.5))
    c.set_spins(mid)
    c.t = 5
    c.step(7)
    assert maxdiff(a.spins(), c.spins()) > 1e-9     # the new field changed the dynamics


def test_magnetisation_oracle():
    s = LT.sc_ferromagnet(4)
    o = O.Oracle(s)
    S = LT.random_spins(s.nspins, 3)
    o.set_spins(S)
    m = o.magnetisation()
    assert np.allclose(m[0, 0], S.mean(axis=0), atol=1e-15)


def test_float_normals_statistics_and_closeness():
    xf = O.thermal_normals_f(11, 3, 20000, 7)
    xd = O.thermal_normals(11, 3, 20000, 7)
    # same 32-bit draw: float and double normals agree to float precision, tails included
    d = np.abs(xf - xd)
    assert d.max() < 2e-6 * max(1.0, np.abs(xd).max())
    v = xf.reshape(-1).astype(np.float64)
    assert abs(v.mean()) < 0.02 and abs(v.var() - 1.0) < 0.03


TS_BIN = os.path.join(os.path.dirname(O.__file__), "_ref", "ref_timeseries")


def _run_ref_timeseries(tmp, series, mesh, sample_dt, width, flo, fhi, hamm=None):
    """Write the reference's k-series and info files, run its analysis tool, read kx*ky*kz*.dat."""
    ns, nk = series.shape
    kp = [(k, 0, 0) for k in range(nk)]
    with open(os.path.join(tmp, "kvec.dat"), "w") as f:
        for t in range(ns):
            f.write(f"{t * sample_dt:.17g}\t" + "".join(f"{z.real:.17g}\t{z.imag:.17g}\t" for z in series[t]) + "\n")
    with open(os.path.join(tmp, "info.in"), "w") as f:
        f.write(f"file: kvec.dat\nsamples: {ns}\ndt: {sample_dt:.17g}\ndim: {mesh[0]} {mesh[1]} {mesh[2]}\n")
        f.write(f"kdim: {mesh[0]} {mesh[1]} {mesh[2]}\nnk: {nk}\n")
        for i, (a, b, c) in enumerate(kp):
            f.write(f"k {i} : {a} {b} {c} x 0 x 0 0 0\n")
    args = [TS_BIN, "info.in", repr(width), repr(flo), repr(fhi)]
    if hamm is not None:
        args += ["hamm", repr(hamm[0]), repr(hamm[1])]
    subprocess.run(args, cwd=tmp, check=True, capture_output=True, timeout=120)
    return [np.loadtxt(os.path.join(tmp, f"kx{a}ky{b}kz{c}.dat")) for a, b, c in kp]


@pytest.mark.skipif(not os.path.exists(TS_BIN), reason="reference time-series tool not built")
@pytest.mark.parametrize("hamm", [None, (0.54, 0.46)])
def test_sq_spectrum_restatement_reproduces_reference_tool(tmp_path, hamm):
    """oracle.sq_spectrum == fourier_space_analysis/src/timeseries.cpp run on the same series
    (window, normalisation, w / ns-1-w pairing, recursive Gaussian, peak search); the tool prints
    6 significant digits."""
    rng = np.random.default_rng(9)
    ns, nk, sdt, mesh = 256, 3, 2e-14, (8, 4, 2)
    t = np.arange(ns) * sdt
    freqs = np.array([3.0e12, 7.5e12, 1.2e13])          # rad/s
    series = (np.exp(-1j * np.outer(t, freqs)) * np.array([5.0, 2.0, 1.0])
              + 0.3 * (rng.normal(size=(ns, nk)) + 1j * rng.normal(size=(ns, nk))))
    width, flo, fhi = 4.0e11, 1.0e11, 1.5e14
    out = _run_ref_timeseries(str(tmp_path), series, mesh, sdt, width, flo, fhi, hamm)
    win = 0 if hamm is None else 1
    # the tool reads alpha from argv[5] (the word "hamm", so 0) and beta from argv[6]
    # (fourier_space_analysis/src/timeseries.cpp:80-81): its window is -hamm[0] cos(2 pi t/(ns-1))
    a, b = (0.54, 0.46) if hamm is None else (0.0, hamm[0])
    raw, sm, pr, ps = O.sq_spectrum(series, np.prod(mesh), win, a, b, width, sdt, flo, fhi)
    for k in range(nk):
        ref = out[k]
        assert ref.shape == (ns // 2, 5)
        np.testing.assert_allclose(ref[:, 0], np.arange(ns // 2) * 2 * np.pi / (ns * sdt), rtol=1e-5)
        np.testing.assert_allclose(ref[:, 1], raw[k], rtol=2e-5, atol=1e-30)
        np.testing.assert_allclose(ref[:, 2], sm[k], rtol=2e-5, atol=1e-30)
        assert ref[pr[k], 3] == 1.0 and ref[ps[k], 4] == 1.0
