"""ctypes binding of the C ABI in include/asd.h (libasd_b200.so, built next to this file).

The binding is a thin layer: every method maps to one asd_* call and raises
AsdError with the library's message on a non-zero status.  There is no CPU
fallback: importing works without a GPU, but creating a handle needs the CUDA
library and a device, and fails loudly otherwise.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libasd_b200.so")

ASD_OK, ASD_EINVAL, ASD_ECUDA, ASD_ENOMEM, ASD_ETIMEOUT, ASD_ESTATE, ASD_ECUFFT, ASD_ENOTSUP, ASD_ENOTFINITE = range(9)
HEUN, RK4, RK5 = 0, 1, 2
FP64_PLAIN, FP32, FP64_FUSED = 0, 1, 2
EXCH_FFT, EXCH_DIA, EXCH_CSR, EXCH_NONE = 0, 1, 2, 3
LR_NONE, LR_DIPOLE, LR_FFT = 0, 1, 2
FLAG_RK_DOUBLE_RDT = 1 << 2
FLAG_RK_STAGE_SPIN_MIXED = 1 << 3
FLAG_GPU_CSR_DIP_STALE = 1 << 4
FLAG_GPU_DZZ_FROM_DYY = 1 << 6
FLAG_GPU_HDEMAG_FP32 = 1 << 7
FLAG_COMPENSATED = 1 << 16
FLAG_AUTOTUNE = 1 << 17
FLAG_STREAMED_EXCHANGE = 1 << 18
FLAG_CUFFT_PLANES = 1 << 19
FLAG_WAIT_TIMEOUT = 1 << 20
FLAG_SERIAL_LAUNCH = 1 << 21
ALL_REPLICAS = 0xFFFFFFFF

MUB, KB, GYRO = 9.27e-24, 1.38e-23, 1.76e11  # reference constants (src/llg.cpp:25)

EXPORTED = [
    "asd_create", "asd_destroy", "asd_last_error", "asd_version", "asd_set_spins", "asd_get_spins",
    "asd_get_det_field", "asd_get_field", "asd_step", "asd_get_step", "asd_set_step", "asd_sync",
    "asd_set_temperature", "asd_set_applied", "asd_set_site_field", "asd_set_site_field_scale",
    "asd_magnetisation", "asd_num_sublattices", "asd_time_steps", "asd_time_kernels", "asd_kernel_stats",
    "asd_thermal_normals", "asd_build_csr", "asd_csr_to_dia", "asd_build_dipole_nr", "asd_fold_exchange_nr",
    "asd_set_site_field_pulse", "asd_sample_magnetisation", "asd_magnetisation_stats",
    "asd_reset_magnetisation_stats", "asd_sq_setup", "asd_sq_sample", "asd_sq_get",
    "asd_sq_spectrum", "asd_tuning", "asd_set_launch_shape",
    "asd_time_kernels_cold", "asd_time_steps_cold", "asd_read_ucf", "asd_read_exch", "asd_read_csr_exch",
    "asd_write_csr_exch", "asd_plan_spin_spans", "asd_set_device_layout", "asd_set_ttm",
    "asd_get_ttm_temperatures", "asd_set_four_spin", "asd_spins_random", "asd_spins_pattern",
    "asd_kernel_table", "asd_get_state", "asd_set_state",
]


class Material(C.Structure):
    _fields_ = [("mu", C.c_double), ("lambda_", C.c_double), ("gamma", C.c_double), ("k1u", C.c_double),
                ("k1u_dir", C.c_double * 3), ("sublattice", C.c_uint32)]


class UcfAtom(C.Structure):
    _fields_ = [("sublattice", C.c_uint32), ("xred", C.c_double * 3), ("mesh_point", C.c_int32 * 3),
                ("mu", C.c_double), ("damping", C.c_double), ("gamma", C.c_double), ("element", C.c_char * 16),
                ("init_spin", C.c_double * 3), ("k1u", C.c_double), ("k1u_dir", C.c_double * 3)]


TTM_MAX_PULSES = 16


class Ttm(C.Structure):
    _fields_ = [("gamma_e", C.c_double), ("Cl", C.c_double), ("G_ep", C.c_double), ("pump_time", C.c_double),
                ("pump_fluence", C.c_double), ("cooling_time", C.c_double), ("initial_T", C.c_double),
                ("npulses", C.c_uint32), ("bath_is_electrons", C.c_uint32),
                ("pulse_scale", C.c_double * TTM_MAX_PULSES), ("pulse_delay", C.c_double * TTM_MAX_PULSES)]


class Params(C.Structure):
    _fields_ = [("integrator", C.c_uint32), ("precision", C.c_uint32), ("dt", C.c_double),
                ("applied", C.c_double * 3), ("k2perp", C.c_double), ("k2perpdir", C.c_double * 3),
                ("k2par", C.c_double), ("k2pardir", C.c_double * 3), ("k4perp", C.c_double),
                ("k4perpdirs", C.c_double * 9), ("k4par", C.c_double), ("k4pardirs", C.c_double * 9),
                ("seed", C.c_uint64), ("update", C.c_uint32), ("flags", C.c_uint32),
                ("gyro", C.c_double), ("muB", C.c_double), ("kB", C.c_double)]


class System(C.Structure):
    _fields_ = [("nspins", C.c_uint32), ("nmat", C.c_uint32), ("mat", C.POINTER(Material)),
                ("atom", C.POINTER(C.c_uint32)), ("exch", C.c_uint32), ("exch_full", C.c_uint32),
                ("xadj", C.POINTER(C.c_uint32)), ("adjncy", C.POINTER(C.c_uint32)), ("nnz", C.c_uint32),
                ("csr_val", C.POINTER(C.c_double)), ("ndiag", C.c_uint32), ("dia_offset", C.POINTER(C.c_int32)),
                ("dia_val", C.POINTER(C.c_double)), ("lr", C.c_uint32), ("mesh", C.c_uint32 * 3),
                ("mesh_xyz", C.POINTER(C.c_uint32)), ("nr", C.POINTER(C.c_double)), ("temperature", C.c_double),
                ("stream", C.c_uint32), ("site_field", C.POINTER(C.c_double))]


class AsdError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"asd error {code}: {msg}")
        self.code = code


_lib = None


def load_library(path: str = LIB_PATH):
    """Load libasd_b200.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} not built: run `make -C {HERE}` (or __graft_entry__.build())")
    lib = C.CDLL(path)
    P = C.c_void_p
    dp = C.POINTER(C.c_double)
    u32p = C.POINTER(C.c_uint32)
    i32p = C.POINTER(C.c_int32)
    sig = {
        "asd_create": ([C.POINTER(Params), C.POINTER(System), C.c_uint32, C.POINTER(P)], C.c_int),
        "asd_destroy": ([P], C.c_int),
        "asd_last_error": ([P], C.c_char_p),
        "asd_version": ([], C.c_char_p),
        "asd_set_spins": ([P, dp, C.c_size_t], C.c_int),
        "asd_get_spins": ([P, dp, C.c_size_t], C.c_int),
        "asd_get_det_field": ([P, dp, C.c_size_t], C.c_int),
        "asd_get_field": ([P, dp, C.c_size_t], C.c_int),
        "asd_step": ([P, C.c_uint64], C.c_int),
        "asd_get_step": ([P, C.POINTER(C.c_uint64)], C.c_int),
        "asd_set_step": ([P, C.c_uint64], C.c_int),
        "asd_sync": ([P], C.c_int),
        "asd_set_temperature": ([P, C.c_uint32, C.c_double], C.c_int),
        "asd_set_applied": ([P, dp], C.c_int),
        "asd_set_site_field": ([P, dp, C.c_size_t], C.c_int),
        "asd_set_site_field_scale": ([P, C.c_double], C.c_int),
        "asd_magnetisation": ([P, dp, C.c_size_t], C.c_int),
        "asd_num_sublattices": ([P, u32p], C.c_int),
        "asd_time_steps": ([P, C.c_uint64, dp, C.POINTER(C.c_uint64)], C.c_int),
        "asd_time_kernels": ([P, C.c_uint64], C.c_int),
        "asd_kernel_stats": ([P, C.c_char_p, C.c_size_t, dp, C.POINTER(C.c_uint64), dp], C.c_int),
        "asd_kernel_table": ([P, C.c_char_p, C.c_size_t], C.c_int),
        "asd_get_state": ([P, C.c_void_p, C.POINTER(C.c_size_t)], C.c_int),
        "asd_set_state": ([P, C.c_void_p, C.c_size_t], C.c_int),
        "asd_thermal_normals": ([C.c_uint64, C.c_uint32, C.c_uint64, C.c_uint32, dp], C.c_int),
        "asd_magnetisation_noalloc": ([C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p],
                                      C.c_int),
        "asd_thermal_normals_f32": ([C.c_uint64, C.c_uint32, C.c_uint64, C.c_uint32, C.POINTER(C.c_float)], C.c_int),
        "asd_set_site_field_pulse": ([P, C.c_double, C.c_double, C.c_double], C.c_int),
        "asd_sample_magnetisation": ([P], C.c_int),
        "asd_magnetisation_stats": ([P, dp, C.c_size_t], C.c_int),
        "asd_reset_magnetisation_stats": ([P], C.c_int),
        "asd_sq_setup": ([P, C.c_uint32, dp, u32p, u32p, C.c_uint32, u32p, C.c_uint32], C.c_int),
        "asd_sq_sample": ([P], C.c_int),
        "asd_sq_get": ([P, dp, C.c_size_t, u32p], C.c_int),
        "asd_tuning": ([P, C.c_char_p, C.c_size_t], C.c_int),
        "asd_read_ucf": ([C.c_char_p, C.c_int, u32p, u32p, C.POINTER(UcfAtom), C.c_uint32, C.c_char_p, C.c_size_t],
                         C.c_int),
        "asd_read_exch": ([C.c_char_p, C.c_uint32, u32p, u32p, u32p, i32p, dp, C.c_uint32, C.c_char_p, C.c_size_t],
                          C.c_int),
        "asd_read_csr_exch": ([C.c_char_p, C.c_uint32, u32p, u32p, u32p, dp, C.c_uint32, C.c_char_p, C.c_size_t],
                              C.c_int),
        "asd_write_csr_exch": ([C.c_char_p, C.c_uint32, u32p, u32p, dp], C.c_int),
        "asd_plan_spin_spans": ([C.c_uint32, C.c_uint32, u32p, u32p, C.c_uint32, C.c_uint32, C.c_uint32, u32p, u32p,
                                 C.c_uint32, u32p, u32p, u32p], C.c_int),
        "asd_time_kernels_cold": ([P, C.c_uint64, C.c_uint64], C.c_int),
        "asd_time_steps_cold": ([P, C.c_uint64, C.c_uint64, dp, C.POINTER(C.c_uint64)], C.c_int),
        "asd_set_launch_shape": ([P, C.c_uint32, C.c_uint32], C.c_int),
        "asd_set_device_layout": ([P, C.c_uint32], C.c_int),
        "asd_set_ttm": ([P, C.c_void_p], C.c_int),
        "asd_set_four_spin": ([P, u32p, u32p, u32p, u32p, C.c_double, C.c_int], C.c_int),
        "asd_get_ttm_temperatures": ([P, dp, dp], C.c_int),
        "asd_sq_spectrum": ([P, C.c_uint32, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                             dp, dp, C.c_size_t, u32p, u32p], C.c_int),
        "asd_build_csr": ([u32p, C.POINTER(C.c_int), C.c_uint32, dp, C.c_uint32, u32p, u32p, i32p, dp, C.c_double,
                           u32p, u32p, dp, u32p], C.c_int),
        "asd_csr_to_dia": ([C.c_uint32, u32p, u32p, dp, C.c_uint32, i32p, dp, u32p], C.c_int),
        "asd_build_dipole_nr": ([u32p, u32p, dp, C.c_double, C.c_double, dp], C.c_int),
        "asd_fold_exchange_nr": ([u32p, C.c_uint32, i32p, dp, C.c_double, dp, u32p], C.c_int),
        "asd_spins_random": ([C.c_uint32, u32p, dp], C.c_int),
        "asd_spins_pattern": ([C.c_uint32, C.c_uint32, i32p, u32p, dp, dp], C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    _lib = lib
    return lib


def _p(a: Optional[np.ndarray], ct):
    if a is None:
        return C.cast(None, C.POINTER(ct))
    return a.ctypes.data_as(C.POINTER(ct))


def _check(rc: int, h=None):
    if rc != ASD_OK:
        msg = ""
        if h is not None:
            m = load_library().asd_last_error(h)
            msg = m.decode() if m else ""
        raise AsdError(rc, msg or "call failed")


@dataclass
class MaterialSpec:
    mu: float = 1.5                 # [muB]
    lam: float = 0.1                # damping
    gamma: float = 1.0              # relative gyromagnetic ratio
    k1u: float = 0.0                # [J/atom]
    k1u_dir: Sequence[float] = (0.0, 0.0, 1.0)
    sublattice: int = 0


@dataclass
class SpinSystem:
    """One lattice with its interactions, in the reference's data contract."""
    nspins: int
    materials: list
    atom: Optional[np.ndarray] = None          # unit-cell atom per spin (None -> i % nmat)
    exch: int = EXCH_NONE
    full: bool = False
    xadj: Optional[np.ndarray] = None
    adjncy: Optional[np.ndarray] = None
    csr_val: Optional[np.ndarray] = None       # nnz x 9 [T]
    dia_offset: Optional[np.ndarray] = None
    dia_val: Optional[np.ndarray] = None       # c x ndiag x n [T], c = 9 if full else 3 (xx,yy,zz)
    lr: int = LR_NONE
    mesh: Sequence[int] = (0, 0, 0)
    mesh_xyz: Optional[np.ndarray] = None      # n x 3
    nr: Optional[np.ndarray] = None            # 9 x P real-space interaction matrix
    temperature: float = 0.0
    stream: int = 0
    site_field: Optional[np.ndarray] = None    # n x 3
    sublattice_of_spin: Optional[np.ndarray] = None
    meta: dict = field(default_factory=dict)

    def nmat(self):
        return len(self.materials)


@dataclass
class RunParams:
    integrator: int = HEUN
    precision: int = FP32
    dt: float = 1e-16
    applied: Sequence[float] = (0.0, 0.0, 0.0)
    k2perp: float = 0.0
    k2perpdir: Sequence[float] = (0.0, 0.0, 0.0)
    k2par: float = 0.0
    k2pardir: Sequence[float] = (0.0, 0.0, 0.0)
    k4perp: float = 0.0
    k4perpdirs: Sequence[float] = (0.0,) * 9
    k4par: float = 0.0
    k4pardirs: Sequence[float] = (0.0,) * 9
    seed: int = 1
    update: int = 1
    flags: int = 0

    def to_c(self) -> Params:
        p = Params()
        p.integrator, p.precision, p.dt = self.integrator, self.precision, self.dt
        p.applied[:] = list(self.applied)
        p.k2perp, p.k2par, p.k4perp, p.k4par = self.k2perp, self.k2par, self.k4perp, self.k4par
        p.k2perpdir[:] = list(self.k2perpdir)
        p.k2pardir[:] = list(self.k2pardir)
        p.k4perpdirs[:] = list(self.k4perpdirs)
        p.k4pardirs[:] = list(self.k4pardirs)
        p.seed, p.update, p.flags = self.seed, self.update, self.flags
        p.gyro, p.muB, p.kB = GYRO, MUB, KB
        return p


class Handle:
    """An asd_handle: one or more replicas advanced together on the current CUDA device."""

    def __init__(self, params: RunParams, systems):
        lib = load_library()
        if isinstance(systems, SpinSystem):
            systems = [systems]
        self._keep = []
        csys = (System * len(systems))()
        for r, s in enumerate(systems):
            mats = (Material * len(s.materials))()
            for t, m in enumerate(s.materials):
                mats[t].mu, mats[t].lambda_, mats[t].gamma, mats[t].k1u = m.mu, m.lam, m.gamma, m.k1u
                mats[t].k1u_dir[:] = list(m.k1u_dir)
                mats[t].sublattice = m.sublattice
            self._keep.append(mats)
            cs = csys[r]
            cs.nspins, cs.nmat, cs.mat = s.nspins, len(s.materials), mats
            arr = lambda a, dt: None if a is None else np.ascontiguousarray(a, dtype=dt)
            atom = arr(s.atom, np.uint32)
            xadj, adj, cv = arr(s.xadj, np.uint32), arr(s.adjncy, np.uint32), arr(s.csr_val, np.float64)
            doff, dval = arr(s.dia_offset, np.int32), arr(s.dia_val, np.float64)
            mxyz, nr, site = arr(s.mesh_xyz, np.uint32), arr(s.nr, np.float64), arr(s.site_field, np.float64)
            self._keep += [atom, xadj, adj, cv, doff, dval, mxyz, nr, site]
            cs.atom = _p(atom, C.c_uint32)
            cs.exch, cs.exch_full = s.exch, 1 if s.full else 0
            cs.xadj, cs.adjncy = _p(xadj, C.c_uint32), _p(adj, C.c_uint32)
            cs.nnz = 0 if adj is None else len(adj)
            cs.csr_val = _p(cv, C.c_double)
            cs.ndiag = 0 if doff is None else len(doff)
            cs.dia_offset, cs.dia_val = _p(doff, C.c_int32), _p(dval, C.c_double)
            cs.lr = s.lr
            cs.mesh[:] = list(s.mesh)
            cs.mesh_xyz, cs.nr = _p(mxyz, C.c_uint32), _p(nr, C.c_double)
            cs.temperature, cs.stream = s.temperature, s.stream
            cs.site_field = _p(site, C.c_double)
        self.params = params
        self.n = sum(s.nspins for s in systems)
        self.nrep = len(systems)
        self._cp = params.to_c()
        h = C.c_void_p()
        rc = lib.asd_create(C.byref(self._cp), csys, len(systems), C.byref(h))
        if rc != ASD_OK:
            raise AsdError(rc, "asd_create failed: " + (lib.asd_last_error(None) or b"").decode(errors="replace"))
        self.h = h
        self._keep = None
        ns = C.c_uint32()
        _check(lib.asd_num_sublattices(self.h, C.byref(ns)), self.h)
        self.nsub = ns.value

    def close(self):
        if getattr(self, "h", None):
            load_library().asd_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_spins(self, s: np.ndarray):
        s = np.ascontiguousarray(s, dtype=np.float64).reshape(-1)
        _check(load_library().asd_set_spins(self.h, _p(s, C.c_double), len(s) // 3), self.h)

    def _read(self, fn, out=None):
        if out is None:
            out = np.empty(3 * self.n, dtype=np.float64)
        if out.dtype != np.float64 or out.size != 3 * self.n or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous float64 array of 3*nspins")
        _check(fn(self.h, _p(out.reshape(-1), C.c_double), self.n), self.h)
        return out.reshape(self.n, 3)

    def get_spins(self, out=None):
        """Spins [n, 3]; `out` (contiguous float64, e.g. pinned host memory) is filled if given."""
        return self._read(load_library().asd_get_spins, out)

    def get_det_field(self):
        return self._read(load_library().asd_get_det_field)

    def get_field(self):
        return self._read(load_library().asd_get_field)

    def step(self, n: int):
        _check(load_library().asd_step(self.h, n), self.h)

    @property
    def t(self) -> int:
        v = C.c_uint64()
        _check(load_library().asd_get_step(self.h, C.byref(v)), self.h)
        return v.value

    def set_step(self, t: int):
        _check(load_library().asd_set_step(self.h, t), self.h)

    def sync(self):
        _check(load_library().asd_sync(self.h), self.h)

    def get_step(self) -> int:
        t = C.c_uint64()
        _check(load_library().asd_get_step(self.h, C.byref(t)), self.h)
        return t.value

    def get_state(self) -> bytes:
        """Exact state (spins in the form's storage, step, bath temperatures, TTM) for restart."""
        lib = load_library()
        n = C.c_size_t()
        _check(lib.asd_get_state(self.h, None, C.byref(n)), self.h)
        buf = C.create_string_buffer(n.value)
        _check(lib.asd_get_state(self.h, buf, C.byref(n)), self.h)
        return buf.raw[: n.value]

    def set_state(self, state: bytes):
        buf = C.create_string_buffer(bytes(state), len(state))
        _check(load_library().asd_set_state(self.h, buf, len(state)), self.h)

    def set_temperature(self, T: float, replica: int = ALL_REPLICAS):
        _check(load_library().asd_set_temperature(self.h, replica, T), self.h)

    def set_applied(self, b):
        a = np.ascontiguousarray(b, dtype=np.float64)
        _check(load_library().asd_set_applied(self.h, _p(a, C.c_double)), self.h)

    def set_site_field(self, prof: Optional[np.ndarray]):
        a = None if prof is None else np.ascontiguousarray(prof, dtype=np.float64).reshape(-1)
        _check(load_library().asd_set_site_field(self.h, _p(a, C.c_double), self.n if a is not None else 0), self.h)

    def set_site_field_scale(self, rv: float):
        _check(load_library().asd_set_site_field_scale(self.h, rv), self.h)

    def set_site_field_pulse(self, amp: float, t0: float, sigma: float):
        _check(load_library().asd_set_site_field_pulse(self.h, amp, t0, sigma), self.h)

    def sample_magnetisation(self):
        _check(load_library().asd_sample_magnetisation(self.h), self.h)

    def magnetisation_stats(self):
        """[replica, sublattice, (samples, mean |m_s|, variance, previous mean)]."""
        out = np.empty(self.nrep * self.nsub * 4, dtype=np.float64)
        _check(load_library().asd_magnetisation_stats(self.h, _p(out, C.c_double), len(out)), self.h)
        return out.reshape(self.nrep, self.nsub, 4)

    def reset_magnetisation_stats(self):
        _check(load_library().asd_reset_magnetisation_stats(self.h), self.h)

    def sq_setup(self, mesh, mesh_xyz, kpoints, max_samples: int, qaxis: int = 2, uo=None):
        """Arm the S(q,t) sampler: spin i sits at mesh_xyz[i] of the lattice mesh; kpoints are
        mesh indices (nk x 3); uo (nsub x 3) are the per-sublattice signs, 1 by default."""
        m = np.ascontiguousarray(mesh, dtype=np.uint32).reshape(3)
        xyz = np.ascontiguousarray(mesh_xyz, dtype=np.uint32).reshape(-1)
        kp = np.ascontiguousarray(kpoints, dtype=np.uint32).reshape(-1)
        u = None if uo is None else np.ascontiguousarray(uo, dtype=np.float64).reshape(-1)
        _check(load_library().asd_sq_setup(self.h, qaxis, _p(u, C.c_double), _p(m, C.c_uint32), _p(xyz, C.c_uint32),
                                           len(kp) // 3, _p(kp, C.c_uint32), max_samples), self.h)
        self._sq_nk = len(kp) // 3
        self._sq_max = max_samples

    def sq_sample(self):
        _check(load_library().asd_sq_sample(self.h), self.h)

    def sq_series(self):
        """psi_k(t) as a complex array [samples, nk]."""
        out = np.empty(self._sq_max * self._sq_nk * 2, dtype=np.float64)
        ns = C.c_uint32()
        _check(load_library().asd_sq_get(self.h, _p(out, C.c_double), len(out), C.byref(ns)), self.h)
        v = out[: ns.value * self._sq_nk * 2].reshape(ns.value, self._sq_nk, 2)
        return v[..., 0] + 1j * v[..., 1]

    def sq_spectrum(self, window=0, alpha=0.54, beta=0.46, width_hz=1.0, sample_dt=1.0, fcut_lo=-np.inf,
                    fcut_hi=np.inf):
        """DSF of the recorded series: raw and smoothed one-sided PSD [nk, ns/2] and the peak bins."""
        ns = self.sq_series().shape[0]
        half = ns // 2
        raw = np.empty(self._sq_nk * half)
        sm = np.empty(self._sq_nk * half)
        pr = np.empty(self._sq_nk, dtype=np.uint32)
        ps = np.empty(self._sq_nk, dtype=np.uint32)
        _check(load_library().asd_sq_spectrum(self.h, window, alpha, beta, width_hz, sample_dt, fcut_lo, fcut_hi,
                                              _p(raw, C.c_double), _p(sm, C.c_double), len(raw),
                                              _p(pr, C.c_uint32), _p(ps, C.c_uint32)), self.h)
        return raw.reshape(self._sq_nk, half), sm.reshape(self._sq_nk, half), pr, ps

    def tuning(self) -> str:
        buf = C.create_string_buffer(512)
        _check(load_library().asd_tuning(self.h, buf, len(buf)), self.h)
        return buf.value.decode()

    def set_ttm(self, gamma_e=None, Cl=None, G_ep=None, pump_time=None, pump_fluence=None, cooling_time=3000e-9,
                initial_T=None, pulses=((1.0, 0.0),), bath_is_electrons=True, off=False):
        """Start (or with off=True stop) the two-temperature model at the current step; pulses are
        (scale, delay [s]) pairs."""
        if off:
            _check(load_library().asd_set_ttm(self.h, None), self.h)
            return
        m = Ttm()
        m.gamma_e, m.Cl, m.G_ep, m.pump_time = gamma_e, Cl, G_ep, pump_time
        m.pump_fluence, m.cooling_time, m.initial_T = pump_fluence, cooling_time, initial_T
        m.npulses, m.bath_is_electrons = len(pulses), int(bath_is_electrons)
        for q, (sc, dl) in enumerate(pulses):
            m.pulse_scale[q], m.pulse_delay[q] = sc, dl
        _check(load_library().asd_set_ttm(self.h, C.byref(m)), self.h)

    def ttm_temperatures(self):
        te, tl = C.c_double(), C.c_double()
        _check(load_library().asd_get_ttm_temperatures(self.h, C.byref(te), C.byref(tl)), self.h)
        return te.value, tl.value

    def set_four_spin(self, xadj, j, k, l, jq, divide_by_3=True):
        """Four-spin quartets (j, k, l) of every spin, CSR over spins; xadj None removes the term."""
        if xadj is None:
            _check(load_library().asd_set_four_spin(self.h, None, None, None, None, 0.0, 0), self.h)
            return
        self._q4 = [np.ascontiguousarray(a, dtype=np.uint32) for a in (xadj, j, k, l)]
        _check(load_library().asd_set_four_spin(self.h, *[_p(a, C.c_uint32) for a in self._q4], jq,
                                                int(divide_by_3)), self.h)

    def set_device_layout(self, layout: int):
        """EXCH_DIA or EXCH_CSR (SELL-32): for a DIA matrix, or a CSR matrix on at most 32 diagonals."""
        _check(load_library().asd_set_device_layout(self.h, layout), self.h)

    def set_launch_shape(self, block: int, staging: int):
        """staging 0: none, 1: typed words, 2: typed words and neighbour spins."""
        _check(load_library().asd_set_launch_shape(self.h, block, int(staging)), self.h)

    def magnetisation(self, out=None):
        if out is None:
            out = np.empty(self.nrep * self.nsub * 3, dtype=np.float64)
        flat = out.reshape(-1)
        _check(load_library().asd_magnetisation(self.h, _p(flat, C.c_double), len(flat)), self.h)
        return out.reshape(self.nrep, self.nsub, 3)

    def time_steps(self, n: int):
        ms = C.c_double()
        l = C.c_uint64()
        _check(load_library().asd_time_steps(self.h, n, C.byref(ms), C.byref(l)), self.h)
        return ms.value, l.value

    def time_steps_cold(self, n: int, flush_bytes: int = 256 << 20):
        """Device ms summed over n steps, each after an untimed L2 flush; and kernel launches."""
        ms = C.c_double()
        l = C.c_uint64()
        _check(load_library().asd_time_steps_cold(self.h, n, flush_bytes, C.byref(ms), C.byref(l)), self.h)
        return ms.value, l.value

    def time_kernels(self, n: int, flush_bytes: int = 0):
        lib = load_library()
        _check(lib.asd_time_kernels_cold(self.h, n, flush_bytes), self.h)
        name = C.create_string_buffer(128)
        avg, cnt, b = C.c_double(), C.c_uint64(), C.c_double()
        _check(lib.asd_kernel_stats(self.h, name, 128, C.byref(avg), C.byref(cnt), C.byref(b)), self.h)
        tab = C.create_string_buffer(8192)
        _check(lib.asd_kernel_table(self.h, tab, len(tab)), self.h)
        kernels = []
        for line in tab.value.decode().splitlines():
            nm, ms, c, by = line.split("|")
            kernels.append({"name": nm, "avg_ms": float(ms), "count": int(c), "bytes": float(by)})
        return {"name": name.value.decode(), "avg_ms": avg.value, "count": cnt.value, "bytes": b.value,
                "kernels": kernels}


def _read_check(rc: int, err):
    if rc != ASD_OK:
        raise AsdError(rc, err.value.decode(errors="replace"))


def read_ucf(path: str, mesh_points: bool = False):
    """Unit-cell file -> (nms, list of per-atom dicts) (geom::readGlobalGeom's .ucf block)."""
    lib = load_library()
    err = C.create_string_buffer(256)
    nms, nauc = C.c_uint32(), C.c_uint32()
    _read_check(lib.asd_read_ucf(path.encode(), int(mesh_points), C.byref(nms), C.byref(nauc), None, 0, err, 256), err)
    atoms = (UcfAtom * nauc.value)()
    _read_check(lib.asd_read_ucf(path.encode(), int(mesh_points), C.byref(nms), C.byref(nauc), atoms, nauc.value,
                                 err, 256), err)
    out = [{"sublattice": a.sublattice, "xred": tuple(a.xred), "mesh_point": tuple(a.mesh_point), "mu": a.mu,
            "damping": a.damping, "gamma": a.gamma, "element": a.element.decode(), "init_spin": tuple(a.init_spin),
            "k1u": a.k1u, "k1u_dir": tuple(a.k1u_dir)} for a in atoms]
    return nms.value, out


def read_exch(path: str, nms: int):
    """Exchange file (libconfig syntax) -> bonds (s1, s2, cell offset (3,), J 3x3 [J]) in file order."""
    lib = load_library()
    err = C.create_string_buffer(256)
    nb = C.c_uint32()
    _read_check(lib.asd_read_exch(path.encode(), nms, C.byref(nb), None, None, None, None, 0, err, 256), err)
    m = max(nb.value, 1)
    s1 = np.zeros(m, dtype=np.uint32)
    s2 = np.zeros(m, dtype=np.uint32)
    v = np.zeros((m, 3), dtype=np.int32)
    J = np.zeros((m, 9))
    _read_check(lib.asd_read_exch(path.encode(), nms, C.byref(nb), _p(s1, C.c_uint32), _p(s2, C.c_uint32),
                                  _p(v, C.c_int32), _p(J, C.c_double), m, err, 256), err)
    k = nb.value
    return s1[:k], s2[:k], v[:k], J[:k].reshape(k, 3, 3)


def read_csr_exch(path: str, nspins: int):
    """csr_exch_mat.dat -> xadj, adjncy, val9 (nnz x 9, diagonal filled)."""
    lib = load_library()
    err = C.create_string_buffer(256)
    nnz = C.c_uint32()
    _read_check(lib.asd_read_csr_exch(path.encode(), nspins, C.byref(nnz), None, None, None, 0, err, 256), err)
    xadj = np.zeros(nspins + 1, dtype=np.uint32)
    adj = np.zeros(nnz.value, dtype=np.uint32)
    val = np.zeros((nnz.value, 9))
    _read_check(lib.asd_read_csr_exch(path.encode(), nspins, C.byref(nnz), _p(xadj, C.c_uint32), _p(adj, C.c_uint32),
                                      _p(val, C.c_double), nnz.value, err, 256), err)
    return xadj, adj, val


def spins_random(n: int, mwc=(1, 101)):
    """spins::setSpinsRandom on the reference's MWC1616 stream seeded (a, b): returns the n x 3
    spins and the stream state after them (to hand on to the next consumer of the stream)."""
    st = np.array(mwc, dtype=np.uint32)
    out = np.zeros((n, 3))
    _check(load_library().asd_spins_random(n, _p(st, C.c_uint32), _p(out, C.c_double)))
    return out, (int(st[0]), int(st[1]))


def spins_pattern(n: int, axis: int, coords=None, atom_of_spin=None, init_spin=None):
    """setSpinsChequerX/Y/Z (axis 0..2, cell coordinates n x 3) or setSpinsConfig (axis 3: the
    initial spin of each spin's unit-cell atom)."""
    c = None if coords is None else np.ascontiguousarray(coords, dtype=np.int32)
    a = None if atom_of_spin is None else np.ascontiguousarray(atom_of_spin, dtype=np.uint32)
    s0 = None if init_spin is None else np.ascontiguousarray(init_spin, dtype=np.float64)
    out = np.zeros((n, 3))
    _check(load_library().asd_spins_pattern(n, axis, _p(c, C.c_int32), _p(a, C.c_uint32), _p(s0, C.c_double),
                                            _p(out, C.c_double)))
    return out


def write_csr_exch(path: str, xadj, adjncy, val9):
    x = np.ascontiguousarray(xadj, dtype=np.uint32)
    a = np.ascontiguousarray(adjncy, dtype=np.uint32)
    v = np.ascontiguousarray(val9, dtype=np.float64)
    _check(load_library().asd_write_csr_exch(path.encode(), len(x) - 1, _p(x, C.c_uint32), _p(a, C.c_uint32),
                                             _p(v, C.c_double)))


def thermal_normals(seed: int, stream: int, step: int, nspins: int) -> np.ndarray:
    out = np.empty(3 * nspins, dtype=np.float64)
    _check(load_library().asd_thermal_normals(seed, stream, step, nspins, _p(out, C.c_double)))
    return out.reshape(nspins, 3)


def thermal_normals_f32(seed: int, stream: int, step: int, nspins: int) -> np.ndarray:
    out = np.empty(3 * nspins, dtype=np.float32)
    _check(load_library().asd_thermal_normals_f32(seed, stream, step, nspins, out.ctypes.data_as(C.POINTER(C.c_float))))
    return out.reshape(nspins, 3)


def version() -> str:
    return load_library().asd_version().decode()
