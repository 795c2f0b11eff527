"""ctypes wrappers of the checkers: liboracle.so (the FP64 CPU restatement) and
_ref/libref_llgcpu*.so (the reference's own llgCPU compiled from source) and
_ref/libref_cuda.so (the reference's own CUDA step kernels compiled from source).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU legs of bench.py; never by the product.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libref_llgcpu.so")
REF_REPLAY_SO = os.path.join(HERE, "_ref", "libref_llgcpu_replay.so")
REF_CUDA_SO = os.path.join(HERE, "_ref", "libref_cuda.so")
REF_SHIM_SO = os.path.join(HERE, "_ref", "libref_shim.so")

CPU_CORRECTOR_ACCUM = 1 << 0
CPU_THERMAL_Z_FROM_X = 1 << 1
RK_DOUBLE_RDT = 1 << 2
RK_STAGE_SPIN_MIXED = 1 << 3
GPU_CSR_DIP_STALE = 1 << 4
CPU_SUM_ORDER = 1 << 5
GPU_DZZ_FROM_DYY = 1 << 6
GPU_HDEMAG_FP32 = 1 << 7
EXCH_NONE, EXCH_DIA, EXCH_CSR = 0, 1, 2
LR_NONE, LR_DIPOLE, LR_FFT = 0, 1, 2
HEUN, RK4, RK5 = 0, 1, 2
NOISE_PHILOX, NOISE_MWC, NOISE_BUFFER = 0, 1, 2
MUB, KB, GYRO = 9.27e-24, 1.38e-23, 1.76e11

dp = C.POINTER(C.c_double)
u32p = C.POINTER(C.c_uint32)
i32p = C.POINTER(C.c_int32)


def reference_dir():
    """The reference tree the checkers compile from: $ASD_REFERENCE_DIR, else the REF default of
    oracle/Makefile (the build recipe names its location)."""
    d = os.environ.get("ASD_REFERENCE_DIR")
    if d:
        return d
    with open(os.path.join(HERE, "Makefile")) as f:
        for line in f:
            if line.startswith("REF ?="):
                return line.split("?=", 1)[1].strip()
    return ""


def build():
    """Compile the checkers (the reference targets only where the reference tree exists)."""
    targets = ["liboracle.so"]
    ref = reference_dir()
    if ref and os.path.isdir(os.path.join(ref, "src")):
        targets.append("ref")
    subprocess.run(["make", "-C", HERE, f"REF={ref}"] + targets, check=True, capture_output=True)


def _ptr(a, ct):
    if a is None:
        return C.cast(None, C.POINTER(ct))
    return a.ctypes.data_as(C.POINTER(ct))


_olib = None


def olib():
    global _olib
    if _olib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = C.CDLL(ORACLE_SO)
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.c_uint32]
        L.orc_destroy.argtypes = [C.c_void_p]
        for name in ["orc_set_material", "orc_set_global_anis", "orc_set_dynamics", "orc_set_replicas",
                     "orc_set_csr", "orc_set_dia", "orc_set_site_field", "orc_set_longrange", "orc_set_flags",
                     "orc_set_noise", "orc_set_spins", "orc_get_spins", "orc_get_det_field", "orc_field", "orc_run",
                     "orc_magnetisation"]:
            getattr(L, name).restype = C.c_int
        L.orc_set_material.argtypes = [C.c_void_p, dp, dp, dp, dp, dp]
        L.orc_set_global_anis.argtypes = [C.c_void_p, C.c_double, dp, C.c_double, dp, C.c_double, dp, C.c_double, dp,
                                          C.c_double]
        L.orc_set_dynamics.argtypes = [C.c_void_p, C.c_int, C.c_double, dp]
        L.orc_set_replicas.argtypes = [C.c_void_p, C.c_uint32, u32p, dp, u32p]
        L.orc_set_csr.argtypes = [C.c_void_p, C.c_int, C.c_uint32, u32p, u32p, dp]
        L.orc_set_dia.argtypes = [C.c_void_p, C.c_int, C.c_uint32, i32p, dp]
        L.orc_set_site_field.argtypes = [C.c_void_p, dp, C.c_double]
        L.orc_set_longrange.argtypes = [C.c_void_p, C.c_int, u32p, u32p, C.c_uint32, u32p, dp, dp, C.c_uint32]
        L.orc_set_flags.argtypes = [C.c_void_p, C.c_uint32]
        L.orc_set_four_spin.restype = C.c_int
        L.orc_set_four_spin.argtypes = [C.c_void_p, u32p, u32p, u32p, u32p, C.c_double, C.c_int]
        L.orc_set_noise.argtypes = [C.c_void_p, C.c_int, C.c_uint64, C.c_uint32, C.c_uint32, dp, C.c_size_t]
        L.orc_set_spins.argtypes = [C.c_void_p, dp]
        L.orc_get_spins.argtypes = [C.c_void_p, dp]
        L.orc_get_det_field.argtypes = [C.c_void_p, dp]
        L.orc_field.argtypes = [C.c_void_p, dp]
        L.orc_run.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64]
        L.orc_magnetisation.argtypes = [C.c_void_p, C.c_uint32, u32p, dp]
        L.orc_philox4x32_10.argtypes = [u32p, u32p, u32p]
        L.orc_thermal_normals.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint64, dp]
        L.orc_log.restype = C.c_double
        L.orc_log.argtypes = [C.c_double]
        L.orc_sincos_2pi.argtypes = [C.c_uint32, dp, dp]
        L.orc_mwc_seed.argtypes = [C.c_uint32, C.c_uint32]
        L.orc_mwc_rand.restype = C.c_double
        L.orc_mwc_normal.restype = C.c_double
        L.orc_csr_to_dia.restype = C.c_int
        L.orc_csr_to_dia.argtypes = [C.c_uint32, u32p, u32p, dp, i32p, dp]
        L.orc_build_dipole_nr.argtypes = [u32p, u32p, dp, C.c_double, C.c_double, dp]
        L.orc_fold_exchange_nr.restype = C.c_int
        L.orc_fold_exchange_nr.argtypes = [u32p, C.c_uint32, i32p, dp, C.c_double, dp]
        _olib = L
    return _olib


def a64(x):
    return None if x is None else np.ascontiguousarray(x, dtype=np.float64)


def au32(x):
    return None if x is None else np.ascontiguousarray(x, dtype=np.uint32)


def expand_dia(s):
    """9-component DIA values (the diagonal form carries xx,yy,zz only)."""
    v = np.asarray(s.dia_val)
    if v.shape[0] == 9:
        return v
    out = np.zeros((9,) + v.shape[1:])
    out[[0, 4, 8]] = v
    return out


class Oracle:
    """FP64 CPU restatement of the step for one handle's worth of spins."""

    def __init__(self, systems, integrator=HEUN, dt=1e-16, applied=(0, 0, 0), flags=0, seed=1, update=1,
                 noise=NOISE_PHILOX, anis=None, noise_buf=None, mwc=(1, 101)):
        if not isinstance(systems, (list, tuple)):
            systems = [systems]
        self.systems = systems
        n = sum(s.nspins for s in systems)
        self.n = n
        L = olib()
        self.c = L.orc_create(n)
        # expand materials per spin (src/llg.cpp:591-592, src/geom.cpp:244)
        llgpf, lam, sig, k1u = (np.zeros(n) for _ in range(4))
        k1d = np.zeros((n, 3))
        off = 0
        sub = np.zeros(n, dtype=np.uint32)
        for s in systems:
            nm = len(s.materials)
            atoms = s.atom if s.atom is not None else np.arange(s.nspins) % nm
            for t, m in enumerate(s.materials):
                sel = off + np.nonzero(atoms == t)[0]
                llgpf[sel] = -1.0 / (1.0 + m.lam * m.lam)
                lam[sel] = m.lam
                sig[sel] = np.sqrt(2.0 * KB * m.lam / (m.mu * MUB * dt * m.gamma * GYRO))
                k1u[sel] = 2.0 * m.k1u / (MUB * m.mu)
                k1d[sel] = m.k1u_dir
                sub[sel] = m.sublattice
            off += s.nspins
        self.sub = sub
        self.nsub = int(sub.max()) + 1
        self._keep = [llgpf, lam, sig, k1u, k1d]
        L.orc_set_material(self.c, _ptr(llgpf, C.c_double), _ptr(lam, C.c_double), _ptr(sig, C.c_double),
                           _ptr(k1u, C.c_double), _ptr(a64(k1d), C.c_double))
        an = anis or {}
        basemm = systems[0].materials[0].mu * MUB
        vec = lambda k, m: a64(an.get(k, [0.0] * m))
        self._an = [vec("k2perpdir", 3), vec("k2pardir", 3), vec("k4perpdirs", 9), vec("k4pardirs", 9)]
        L.orc_set_global_anis(self.c, an.get("k2perp", 0.0), _ptr(self._an[0], C.c_double), an.get("k2par", 0.0),
                              _ptr(self._an[1], C.c_double), an.get("k4perp", 0.0), _ptr(self._an[2], C.c_double),
                              an.get("k4par", 0.0), _ptr(self._an[3], C.c_double), basemm)
        ap = a64(applied)
        self._integrator, self._rdt = integrator, dt * GYRO
        L.orc_set_dynamics(self.c, integrator, dt * GYRO, _ptr(ap, C.c_double))
        roff = au32(np.concatenate([[0], np.cumsum([s.nspins for s in systems])]))
        T = a64([s.temperature for s in systems])
        st = au32([s.stream for s in systems])
        self._off, self._T, self._stream = roff, T, st
        L.orc_set_replicas(self.c, len(systems), _ptr(roff, C.c_uint32), _ptr(T, C.c_double), _ptr(st, C.c_uint32))
        s0 = systems[0]
        if s0.exch == 2:  # CSR (asd_b200.EXCH_CSR)
            xs, ads, vs = [np.zeros(1, dtype=np.uint32)], [], []
            base = 0
            for r, s in enumerate(systems):
                xs.append(s.xadj[1:] + base)
                ads.append(s.adjncy + roff[r])
                vs.append(s.csr_val)
                base += len(s.adjncy)
            xadj = au32(np.concatenate(xs))
            adj = au32(np.concatenate(ads))
            val = a64(np.concatenate(vs))
            self._keep += [xadj, adj, val]
            L.orc_set_csr(self.c, 1 if s0.full else 0, len(adj), _ptr(xadj, C.c_uint32), _ptr(adj, C.c_uint32),
                          _ptr(val, C.c_double))
        elif s0.exch == 1:  # DIA
            doff = np.ascontiguousarray(s0.dia_offset, dtype=np.int32)
            dval = a64(expand_dia(s0))
            self._keep += [doff, dval]
            L.orc_set_dia(self.c, 1 if s0.full else 0, len(doff), _ptr(doff, C.c_int32), _ptr(dval, C.c_double))
        if s0.site_field is not None:
            hs = a64(np.concatenate([s.site_field if s.site_field is not None else np.zeros((s.nspins, 3))
                                     for s in systems]))
            self._keep.append(hs)
            L.orc_set_site_field(self.c, _ptr(hs, C.c_double), 1.0)
        if s0.lr:
            mesh = au32(s0.mesh)
            mxyz = au32(s0.mesh_xyz)
            nr = a64(s0.nr)
            atoms = s0.atom if s0.atom is not None else np.arange(s0.nspins) % len(s0.materials)
            w = a64([s0.materials[a].mu for a in atoms]) if s0.lr == LR_DIPOLE else None
            self._keep += [mesh, mxyz, nr, w]
            L.orc_set_longrange(self.c, s0.lr, _ptr(mesh, C.c_uint32), _ptr(mxyz, C.c_uint32), 1, None,
                                _ptr(nr, C.c_double), _ptr(w, C.c_double), update)
        L.orc_set_flags(self.c, flags)
        nb = a64(noise_buf)
        L.orc_set_noise(self.c, noise, seed, mwc[0], mwc[1], _ptr(nb, C.c_double), 0 if nb is None else len(nb))
        self.t = 0

    def __del__(self):
        try:
            olib().orc_destroy(self.c)
        except Exception:
            pass

    def set_four_spin(self, xadj, j, k, l, jq, div3=True):
        L = olib()
        self._q4 = [au32(xadj), au32(j), au32(k), au32(l)]
        L.orc_set_four_spin(self.c, *[_ptr(a, C.c_uint32) for a in self._q4], C.c_double(jq), int(div3))

    def set_temperatures(self, T):
        """Replica temperatures [K] for the following steps (the spin bath of a driver that changes
        T between steps)."""
        L = olib()
        self._T = a64(T)
        L.orc_set_replicas(self.c, len(self._T), _ptr(self._off, C.c_uint32), _ptr(self._T, C.c_double),
                           _ptr(self._stream, C.c_uint32))

    def set_pulse(self, amp, t0, sigma, dt):
        L = olib()
        L.orc_set_pulse.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_double]
        L.orc_set_pulse(self.c, amp, t0, sigma, dt)

    def set_site_scale(self, rv):
        hs = a64(np.concatenate([s.site_field for s in self.systems]))
        self._keep.append(hs)
        olib().orc_set_site_field(self.c, _ptr(hs, C.c_double), rv)

    def set_spins(self, s):
        s = a64(s).reshape(-1)
        olib().orc_set_spins(self.c, _ptr(s, C.c_double))

    def spins(self):
        out = np.empty(3 * self.n)
        olib().orc_get_spins(self.c, _ptr(out, C.c_double))
        return out.reshape(self.n, 3)

    def det_field(self):
        out = np.empty(3 * self.n)
        olib().orc_get_det_field(self.c, _ptr(out, C.c_double))
        return out.reshape(self.n, 3)

    def field(self):
        out = np.empty(3 * self.n)
        olib().orc_field(self.c, _ptr(out, C.c_double))
        return out.reshape(self.n, 3)

    def step(self, k):
        olib().orc_run(self.c, self.t, k)
        self.t += k

    def set_applied(self, b):
        """The applied field from the next step on, as the reference's field ramp sets
        llg::applied between steps (src/ramp_field.cpp:221-223)."""
        ap = a64(b)
        olib().orc_set_dynamics(self.c, self._integrator, self._rdt, _ptr(ap, C.c_double))

    def magnetisation(self):
        out = np.empty(len(self.systems) * self.nsub * 3)
        sub = au32(self.sub)
        olib().orc_magnetisation(self.c, self.nsub, _ptr(sub, C.c_uint32), _ptr(out, C.c_double))
        return out.reshape(len(self.systems), self.nsub, 3)


def philox(ctr, key):
    c = au32(ctr)
    k = au32(key)
    o = np.zeros(4, dtype=np.uint32)
    olib().orc_philox4x32_10(_ptr(c, C.c_uint32), _ptr(k, C.c_uint32), _ptr(o, C.c_uint32))
    return o


def thermal_normals_f(seed, stream, n, step):
    """The FP32 form's normals (single-precision series on the same Philox draw)."""
    L = olib()
    L.orc_thermal_normals_f.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint64, C.POINTER(C.c_float)]
    out = np.zeros((n, 3), dtype=np.float32)
    buf = (C.c_float * 3)()
    for i in range(n):
        L.orc_thermal_normals_f(seed, stream, i, step, buf)
        out[i] = buf[:]
    return out


def thermal_normals(seed, stream, n, step):
    out = np.zeros((n, 3))
    L = olib()
    buf = (C.c_double * 3)()
    for i in range(n):
        L.orc_thermal_normals(seed, stream, i, step, buf)
        out[i] = buf[:]
    return out


class RefLLGCPU:
    """The reference's own llgCPU::llgCPU (src/llgCPU.cpp:56-361) behind ref_harness.cpp."""

    def __init__(self, system, dt=1e-16, applied=(0, 0, 0), replay=False, seed=(1, 101), path=None,
                 anis=None):
        path = path or (REF_REPLAY_SO if replay else REF_SO)
        if not os.path.exists(path):
            build()
        # each instance gets its own copy of the globals: load a private copy of the library
        self.L = C.CDLL(path, mode=os.RTLD_LOCAL)
        L = self.L
        L.refh_init.argtypes = [C.c_uint, C.c_uint, dp, dp, dp, u32p, C.c_double, C.c_double, dp]
        L.refh_set_anis.argtypes = [dp, dp, C.c_double, dp, C.c_double, dp, C.c_double, dp, C.c_double, dp]
        L.refh_set_csr.argtypes = [C.c_int, C.c_uint, u32p, u32p, dp]
        L.refh_set_dia.argtypes = [C.c_int, C.c_uint, i32p, dp, C.c_uint]
        L.refh_set_site_fields.argtypes = [dp, dp]
        L.refh_set_spins.argtypes = [dp]
        L.refh_get_spins.argtypes = [dp]
        L.refh_get_field.argtypes = [dp]
        L.refh_seed.argtypes = [C.c_uint, C.c_uint]
        L.refh_run.argtypes = [C.c_uint, C.c_uint]
        L.refh_set_temperature.argtypes = [C.c_double]
        L.refh_normal.restype = C.c_double
        if replay:
            L.refh_set_noise.argtypes = [dp, C.c_size_t]
        s = system
        self.n = s.nspins
        mats = s.materials
        mu = a64([m.mu for m in mats])
        lam = a64([m.lam for m in mats])
        gam = a64([m.gamma for m in mats])
        atoms = au32(s.atom if s.atom is not None else np.arange(s.nspins) % len(mats))
        ap = a64(applied)
        L.refh_init(s.nspins, len(mats), _ptr(mu, C.c_double), _ptr(lam, C.c_double), _ptr(gam, C.c_double),
                    _ptr(atoms, C.c_uint32), dt, s.temperature, _ptr(ap, C.c_double))
        k1u = a64([2.0 * mats[a].k1u / (MUB * mats[a].mu) for a in atoms])
        k1d = a64([mats[a].k1u_dir for a in atoms])
        # anis: the global K2/K4 terms in J as in anis:: (k2perp, k2perpdir, k2par, k2pardir,
        # k4perp, k4perpdirs[3][3], k4par, k4pardirs[3][3])
        a = dict(anis or {})
        dirs = {k: a64(a.get(k, np.zeros(9 if k.startswith("k4") else 3))).reshape(-1)
                for k in ("k2perpdir", "k2pardir", "k4perpdirs", "k4pardirs")}
        self._anis = dirs
        L.refh_set_anis(_ptr(k1u, C.c_double), _ptr(k1d, C.c_double),
                        float(a.get("k2perp", 0.0)), _ptr(dirs["k2perpdir"], C.c_double),
                        float(a.get("k2par", 0.0)), _ptr(dirs["k2pardir"], C.c_double),
                        float(a.get("k4perp", 0.0)), _ptr(dirs["k4perpdirs"], C.c_double),
                        float(a.get("k4par", 0.0)), _ptr(dirs["k4pardirs"], C.c_double))
        if s.exch == 2:
            xadj, adj, val = au32(s.xadj), au32(s.adjncy), a64(s.csr_val)
            self._keep = [xadj, adj, val]
            L.refh_set_csr(1 if s.full else 0, len(adj), _ptr(xadj, C.c_uint32), _ptr(adj, C.c_uint32),
                           _ptr(val, C.c_double))
        elif s.exch == 1:
            off = np.ascontiguousarray(s.dia_offset, dtype=np.int32)
            val = a64(expand_dia(s))
            self._keep = [off, val]
            L.refh_set_dia(1 if s.full else 0, len(off), _ptr(off, C.c_int32), _ptr(val, C.c_double),
                           len(off))
        if s.site_field is not None:
            hs = a64(s.site_field)
            self._keep.append(hs)
            L.refh_set_site_fields(_ptr(hs, C.c_double), None)
        if not replay and path != REF_CUDA_SO:
            L.refh_seed(*seed)
        self.t = 0

    def set_four_spin(self, xadj, j, k, l, jq):
        """Quartets as exch::xadj_j / adjncy_j,k,l and JQ(0) [T] (src/exch_read_4_spin.cpp)."""
        q = [au32(a) for a in (xadj, j, k, l)]
        self._q4 = q
        self.L.refh_set_four_spin.argtypes = [C.c_uint, u32p, u32p, u32p, u32p, C.c_double]
        self.L.refh_set_four_spin(len(q[1]), *[_ptr(a, C.c_uint32) for a in q], float(jq))

    def set_noise(self, xi):
        x = a64(xi).reshape(-1)
        self._noise = x
        self.L.refh_set_noise(_ptr(x, C.c_double), len(x))

    def set_spins(self, s):
        s = a64(s).reshape(-1)
        self.L.refh_set_spins(_ptr(s, C.c_double))

    def spins(self):
        out = np.empty(3 * self.n)
        self.L.refh_get_spins(_ptr(out, C.c_double))
        return out.reshape(self.n, 3)

    def step(self, k):
        rc = self.L.refh_run(self.t, k)
        self.t += k
        return rc


class RefCUDA(RefLLGCPU):
    """The reference's own CUDA step kernels (CHeun1/2, CSpMV_*, CdetRK4k*/RK5k*, src/cuint.cu,
    src/cufields.cu, src/cuintRK4.cu, src/cuintRK5.cu) launched in the order of src/cuda.cu:43-258,
    src/cudaRK4.cu:38-233 and src/cudaRK5.cu, behind ref_cuda_harness.cu.  Needs a GPU.  The
    globals are filled exactly as for RefLLGCPU; set_spins() uploads everything, so call the
    setters (four-spin, temperature) before it.  Crand (float normals) is set by the caller and
    reused by every step until set again."""

    def __init__(self, system, dt=1e-16, applied=(0, 0, 0), integrator=HEUN, block=128, dzz_from_dyy=False,
                 anis=None):
        super().__init__(system, dt=dt, applied=applied, path=REF_CUDA_SO, anis=anis)
        L = self.L
        L.refg_init.argtypes = [C.c_uint, C.c_int]
        L.refg_set_noise.argtypes = [C.POINTER(C.c_float), C.c_size_t]
        L.refg_run.argtypes = [C.c_int, C.c_uint]
        L.refg_get_spins.argtypes = [dp]
        L.refg_get_det_field.argtypes = [dp]
        self.integrator, self.block, self.dzz = integrator, block, bool(dzz_from_dyy)

    def set_spins(self, s):
        super().set_spins(s)
        rc = self.L.refg_init(self.block, 1 if self.dzz else 0)
        if rc != 0:
            raise RuntimeError(f"refg_init failed ({rc})")

    def set_noise(self, xi):
        x = np.ascontiguousarray(np.asarray(xi, dtype=np.float32).reshape(-1))
        rc = self.L.refg_set_noise(_ptr(x, C.c_float), len(x))
        if rc != 0:
            raise RuntimeError(f"refg_set_noise failed ({rc})")

    def step(self, k):
        rc = self.L.refg_run(self.integrator, k)
        if rc != 0:
            raise RuntimeError(f"refg_run failed ({rc})")
        self.t += k
        return rc

    def spins(self):
        out = np.empty(3 * self.n)
        self.L.refg_get_spins(_ptr(out, C.c_double))
        return out.reshape(self.n, 3)

    def det_field(self):
        out = np.empty(3 * self.n)
        self.L.refg_get_det_field(_ptr(out, C.c_double))
        return out.reshape(self.n, 3)

    def buffer(self, which):
        """Work array after the last step: 0..5 CRKk1..6, 6 Cespin, 7 CH."""
        out = np.empty(3 * self.n)
        self.L.refg_get_buffer.argtypes = [C.c_int, dp]
        self.L.refg_get_buffer(which, _ptr(out, C.c_double))
        return out.reshape(self.n, 3)

    def enable_curand(self, seed):
        """Draw Crand with cuRAND XORWOW every step, seeded as cullg::cuinit does (src/cuda.cu:345-368)."""
        self.L.refg_enable_curand.argtypes = [C.c_ulonglong]
        if self.L.refg_enable_curand(seed) != 0:
            raise RuntimeError("refg_enable_curand failed")

    def time_steps_cold(self, nsteps, flush_bytes=256 << 20):
        """Device ms of nsteps Heun steps, each after an untimed L2 flush, CUDA events per step."""
        ms = C.c_double()
        self.L.refg_time_steps.argtypes = [C.c_int, C.c_uint, C.c_size_t, dp]
        rc = self.L.refg_time_steps(self.integrator, nsteps, flush_bytes, C.byref(ms))
        if rc != 0:
            raise RuntimeError(f"refg_time_steps failed ({rc})")
        return ms.value

    def close(self):
        self.L.refg_free()


class RefShim(RefLLGCPU):
    """The library driven through the reference-side binding gpu-atomistic-code_b200/shim/cullg_asd.cpp:
    the reference's namespace globals are filled as for RefLLGCPU, then cullg::cuinit and
    cullg::llgGPU / llgGPURK4 / llgGPURK5 run as llg::integrate calls them; spins are read back
    from the spins::Sx/Sy/Sz mirror the shim refreshes every `update` steps.  Needs a GPU."""

    def __init__(self, system, dt=1e-16, applied=(0, 0, 0), integrator=HEUN, precision=2, flags=0, seed=1,
                 update=1, anis=None):
        super().__init__(system, dt=dt, applied=applied, path=REF_SHIM_SO, anis=anis)
        L = self.L
        s = system
        atoms = au32(s.atom if s.atom is not None else np.arange(s.nspins) % len(s.materials))
        coords = np.zeros((s.nspins, 3), dtype=np.int32)
        L.refs_set_lu.argtypes = [C.c_uint, u32p, i32p]
        L.refs_set_ucm.argtypes = [C.c_uint, dp, dp, u32p]
        L.refs_configure.argtypes = [C.c_uint] * 5
        L.refs_run.argtypes = [C.c_uint, C.c_uint]
        L.refs_set_lu(s.nspins, _ptr(atoms, C.c_uint32), _ptr(coords, C.c_int32))
        k1u = a64([m.k1u for m in s.materials])
        dirs = a64([m.k1u_dir for m in s.materials]).reshape(-1)
        sub = au32([m.sublattice for m in s.materials])
        L.refs_set_ucm(len(s.materials), _ptr(k1u, C.c_double), _ptr(dirs, C.c_double), _ptr(sub, C.c_uint32))
        L.refs_configure(integrator, seed, update, precision, flags)
        self._keep_shim = [atoms, coords, k1u, dirs, sub]

    def _check(self, what):
        self.L.refh_last_error.restype = C.c_char_p
        msg = self.L.refh_last_error().decode()
        if msg:
            raise RuntimeError(f"{what}: {msg}")

    def set_spins(self, s):
        super().set_spins(s)
        self.L.refs_cuinit()
        self._check("cullg::cuinit")

    def step(self, k):
        self.L.refs_run(self.t, k)
        self._check("cullg::llgGPU")
        self.t += k
        return 0

    def close(self):
        self.L.refs_free()


def spins_random(n, mwc=(1, 101)):
    """spins::setSpinsRandom (src/spins.cpp:265-281): Marsaglia's point on the sphere, v1, v2 =
    2 rand - 1 until v1^2 + v2^2 <= 1, S = (2 v1 sqrt(1-s), 2 v2 sqrt(1-s), 1 - 2 s), with
    rand() the oracle's MWC1616 (src/random.cpp:17-40)."""
    L = olib()
    L.orc_mwc_seed(int(mwc[0]), int(mwc[1]))
    out = np.zeros((n, 3))
    for i in range(n):
        v1 = v2 = 0.0
        s = 2.0
        while s > 1.0:
            v1 = 2.0 * L.orc_mwc_rand() - 1.0
            v2 = 2.0 * L.orc_mwc_rand() - 1.0
            s = v1 * v1 + v2 * v2
        ss = math.sqrt(1.0 - s)
        out[i] = (2.0 * v1 * ss, 2.0 * v2 * ss, 1.0 - 2.0 * s)
    return out


def ref_rand_stream(k, mwc=(1, 101)):
    """k values of the reference's own Random::rand (src/random.cpp:37-40), compiled from source."""
    if not os.path.exists(REF_SO):
        build()
    L = C.CDLL(REF_SO, mode=os.RTLD_LOCAL)
    L.refh_seed.argtypes = [C.c_uint, C.c_uint]
    L.refh_rand.restype = C.c_double
    L.refh_seed(int(mwc[0]), int(mwc[1]))
    return np.array([L.refh_rand() for _ in range(k)])


def sq_psi_k(S, sub, uo, mesh, mesh_xyz, kpoints, qaxis=2):
    """psi_k of one sample: psi = uo_a S_a + i uo_b S_b on the mesh (a, b transverse to the
    quantisation axis), forward 3D FFT (FFTW sign), values at the k-points
    (src/timeseries.cpp:280-314)."""
    a, b = (1, 2) if qaxis == 0 else ((0, 2) if qaxis == 1 else (0, 1))
    uo = np.asarray(uo, dtype=np.float64)
    xyz = np.asarray(mesh_xyz, dtype=np.int64)
    kp = np.asarray(kpoints, dtype=np.int64)
    g = np.zeros(tuple(mesh), dtype=np.complex128)
    g[xyz[:, 0], xyz[:, 1], xyz[:, 2]] = S[:, a] * uo[sub, a] + 1j * (S[:, b] * uo[sub, b])
    return np.fft.fftn(g)[kp[:, 0], kp[:, 1], kp[:, 2]]


def gaussian_iir(x, sigma, nsteps=10):
    """Recursive Gaussian of Alvarez and Mazorra (SIAM J. Numer. Anal. 31, 590, 1994) as the
    time-series tool applies it (fourier_space_analysis/src/timeseries.cpp:289-325)."""
    d = np.array(x, dtype=np.float64)
    n = len(d)
    lam = (sigma * sigma) / (2.0 * nsteps)
    nu = (1.0 + 2.0 * lam - np.sqrt(1.0 + 4.0 * lam)) / (2.0 * lam)
    bscale = 1.0 / (1.0 - nu)
    post = (nu / lam) ** nsteps
    for _ in range(nsteps):
        d[0] *= bscale
        for i in range(1, n):
            d[i] += nu * d[i - 1]
        d[n - 1] *= bscale
        for i in range(n - 1, 0, -1):
            d[i - 1] += nu * d[i]
    return d * post


def sq_spectrum(series, mesh_points, window=0, alpha=0.54, beta=0.46, width_hz=1.0, sample_dt=1.0,
                fcut_lo=-np.inf, fcut_hi=np.inf):
    """Per-k-point DSF of a psi_k(t) series [ns, nk] (fourier_space_analysis/src/timeseries.cpp:142-275):
    optional generalised Hamming window, forward FFT in time divided by mesh_points*ns, one-sided
    PSD pairing w with ns-1-w, Gaussian smoothing of round(width*ns*dt) bins, peak search inside
    the frequency cut (raw peak from w > 1).  Returns raw, smooth [nk, ns/2], peak_raw, peak_smooth."""
    ns, nk = series.shape
    x = np.array(series, dtype=np.complex128)
    if window == 1:
        t = np.arange(ns, dtype=np.float64)
        x = x * (alpha - beta * np.cos(2.0 * np.pi * t / (ns - 1.0)))[:, None]
    X = np.fft.fft(x, axis=0) / (float(mesh_points) * ns)
    half = ns // 2
    w = np.arange(half)
    raw = (np.abs(X[w]) ** 2 + np.abs(X[ns - 1 - w]) ** 2).T
    pw = int(width_hz * ns * sample_dt + 0.5)
    smooth = np.stack([gaussian_iir(r, float(pw)) for r in raw])
    f = w * 2.0 * np.pi / (ns * sample_dt)
    inside = (f > fcut_lo) & (f < fcut_hi)
    pr = np.zeros(nk, dtype=np.uint32)
    ps = np.zeros(nk, dtype=np.uint32)
    for k in range(nk):
        mr = ms = 0.0
        for i in range(half):
            if smooth[k, i] > ms and inside[i]:
                ms, ps[k] = smooth[k, i], i
            if raw[k, i] > mr and i > 1 and inside[i]:
                mr, pr[k] = raw[k, i], i
    return raw, smooth, pr, ps


REF_BUILDERS_SO = os.path.join(HERE, "_ref", "libref_builders.so")


def _ref_builders():
    if not os.path.exists(REF_BUILDERS_SO):
        build()
    L = C.CDLL(REF_BUILDERS_SO, mode=os.RTLD_LOCAL)
    L.refb_exchunitcell.argtypes = [u32p, C.POINTER(C.c_int), C.c_uint, dp, u32p, C.c_uint, dp, dp, C.c_int,
                                    u32p, u32p, u32p, dp, C.c_uint]
    L.refb_csr_to_dia.argtypes = [C.c_uint, u32p, u32p, dp, C.c_int, u32p, i32p, dp, C.c_uint]
    return L


def ref_exchunitcell(dim, pbc, mus, bonds, offdiag=True):
    """The reference's exch::exchunitcell (src/exch_unitcell.cpp:265-489) on bonds given as
    (atom s1, atom s2, cell offset, 3x3 J [J]) in shell order per (s1, s2).  Returns xadj,
    adjncy, val9 (J/(mu muB), nnz x 9; only xx, yy, zz unless offdiag)."""
    L = _ref_builders()
    nauc = len(mus)
    per = {}
    for s1, s2, v, Jm in bonds:
        per.setdefault((s1, s2), []).append((v, np.asarray(Jm, dtype=np.float64).reshape(9)))
    maxsh = max([len(x) for x in per.values()] + [1])
    shells = np.zeros(nauc * nauc, dtype=np.uint32)
    vec = np.zeros((nauc * nauc * maxsh, 3))
    Jt = np.zeros((nauc * nauc * maxsh, 9))
    for (s1, s2), lst in per.items():
        shells[s1 * nauc + s2] = len(lst)
        for k, (v, Jm) in enumerate(lst):
            vec[(s1 * nauc + s2) * maxsh + k] = v
            Jt[(s1 * nauc + s2) * maxsh + k] = Jm
    d = au32(dim)
    p = np.ascontiguousarray(pbc, dtype=np.int32)
    m = a64(mus)
    nnz = C.c_uint()
    args = [_ptr(d, C.c_uint32), p.ctypes.data_as(C.POINTER(C.c_int)), nauc, _ptr(m, C.c_double),
            _ptr(shells, C.c_uint32), maxsh, _ptr(vec, C.c_double), _ptr(Jt, C.c_double), int(offdiag)]
    L.refb_exchunitcell(*args, C.byref(nnz), None, None, None, 0)
    n = int(np.prod(dim)) * nauc
    xadj = np.zeros(n + 1, dtype=np.uint32)
    adj = np.zeros(max(nnz.value, 1), dtype=np.uint32)
    val = np.zeros((max(nnz.value, 1), 9))
    rc = L.refb_exchunitcell(*args, C.byref(nnz), _ptr(xadj, C.c_uint32), _ptr(adj, C.c_uint32),
                             _ptr(val, C.c_double), len(adj))
    assert rc == 0
    return xadj, adj[: nnz.value], val[: nnz.value]


def ref_csr_to_dia(n, xadj, adjncy, val9, offdiag=True):
    """The reference's matconv::csr_to_dia_diag / _offdiag (src/matrix_conv.cpp:28-272).
    Returns offsets and data [9, ndiag*n] (row-aligned, component-major)."""
    L = _ref_builders()
    x, a, v = au32(xadj), au32(adjncy), a64(val9)
    nd = C.c_uint()
    L.refb_csr_to_dia(n, _ptr(x, C.c_uint32), _ptr(a, C.c_uint32), _ptr(v, C.c_double), int(offdiag), C.byref(nd),
                      None, None, 0)
    off = np.zeros(nd.value, dtype=np.int32)
    data = np.zeros(9 * nd.value * n)
    rc = L.refb_csr_to_dia(n, _ptr(x, C.c_uint32), _ptr(a, C.c_uint32), _ptr(v, C.c_double), int(offdiag),
                           C.byref(nd), _ptr(off, C.c_int32), _ptr(data, C.c_double), nd.value)
    assert rc == 0
    return off, data.reshape(9, nd.value * n)


def ttm_step(state, prm, step, dt):
    """One two-temperature-model step, src/laser_heating.cpp:884-895 (CalcTe): the electron
    temperature first, then the lattice with the new Te.  state = [Te, Tl] is updated in place;
    prm: gamma_e, Cl, G_ep, pump_time, pump_fluence, cooling_time, initial_T, pulses, t0 (start
    step).  Returns the bath temperature (Te or Tl)."""
    time = (step - prm["t0"]) * dt
    P = 0.0
    for sc, dl in prm["pulses"]:
        x = (time - dl) / prm["pump_time"]
        P += prm["pump_fluence"] * sc * math.exp(-(x * x))
    Te, Tl = state
    G, Cl = prm["G_ep"], prm["Cl"]
    Te_n = (-G * (Te - Tl) + P) * dt / (prm["gamma_e"] * Te) + Te
    Tl_n = (G * (Te_n - Tl) - Cl * (Tl - prm["initial_T"]) / prm["cooling_time"]) * dt / Cl + Tl
    state[0], state[1] = Te_n, Tl_n
    return Te_n if prm.get("bath_is_electrons", True) else Tl_n
