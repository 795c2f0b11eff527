"""Lattice, exchange and interaction-matrix set-up (the reference's geom/exch/intmat layer).

Everything here is set-up work on the host in FP64, done through the library's
C-ABI builders (asd_build_csr, asd_csr_to_dia, asd_build_dipole_nr,
asd_fold_exchange_nr).  The workload constructors reproduce the lattices the
benchmark configurations describe, with seeded synthetic parameters:

  sc_ferromagnet      simple cubic, nearest-neighbour isotropic exchange (CSR), optional dipole
  bct2_antiferromagnet body-centred tetragonal, 2 sublattices, 4 shells / 26 neighbours,
                      full 3x3 tensors with antisymmetric (DMI-like) parts, CSR or DIA
  sc_fft              simple cubic, open boundaries, dipole + exchange folded into N_k
  film_dia            thin film, J1+J2 in DIA, optional dipole, site-field pulse profile
  replica_batch       uneven sc replicas with their own temperature and Philox stream
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Optional, Sequence

import numpy as np

import asd_b200 as A

J_SC = 1e-21          # [J]
MU_SC = 1.5           # [muB]
K1U_SC = 1e-23        # [J/atom]


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def random_spins(n: int, seed: int) -> np.ndarray:
    """Unit vectors uniform on the sphere: z ~ U[-1,1), phi ~ U[0,2pi) from numpy PCG64(seed)."""
    rng = np.random.default_rng(seed)
    z = rng.uniform(-1.0, 1.0, n)
    phi = rng.uniform(0.0, 2.0 * math.pi, n)
    r = np.sqrt(1.0 - z * z)
    return np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=1)


def build_csr(dim, pbc, mus, bond_atom, bond_to, bond_vec, bond_J):
    """Bond list -> CSR (values J/(mu muB) [T]) via asd_build_csr."""
    lib = A.load_library()
    dim = _u32(dim)
    pbc = np.ascontiguousarray(pbc, dtype=np.int32)
    mus = np.ascontiguousarray(mus, dtype=np.float64)
    ba, bt = _u32(bond_atom), _u32(bond_to)
    bv = np.ascontiguousarray(bond_vec, dtype=np.int32).reshape(-1)
    bj = np.ascontiguousarray(bond_J, dtype=np.float64).reshape(-1)
    nb = len(ba)
    nnz = C.c_uint32()
    args = [A._p(dim, C.c_uint32), pbc.ctypes.data_as(C.POINTER(C.c_int)), len(mus), A._p(mus, C.c_double), nb,
            A._p(ba, C.c_uint32), A._p(bt, C.c_uint32), A._p(bv, C.c_int32), A._p(bj, C.c_double), A.MUB]
    A._check(lib.asd_build_csr(*args, None, None, None, C.byref(nnz)))
    n = int(np.prod(dim)) * len(mus)
    xadj = np.zeros(n + 1, dtype=np.uint32)
    adj = np.zeros(max(nnz.value, 1), dtype=np.uint32)
    val = np.zeros((max(nnz.value, 1), 9), dtype=np.float64)
    A._check(lib.asd_build_csr(*args, A._p(xadj, C.c_uint32), A._p(adj, C.c_uint32), A._p(val, C.c_double),
                               C.byref(nnz)))
    return xadj, adj[: nnz.value], val[: nnz.value]


def csr_to_dia(n, xadj, adjncy, val9, ncomp=9):
    """CSR -> row-aligned DIA with ncomp (3: xx,yy,zz; 9: full) components per diagonal entry."""
    lib = A.load_library()
    xadj, adjncy = _u32(xadj), _u32(adjncy)
    val9 = np.ascontiguousarray(val9, dtype=np.float64)
    nd = C.c_uint32()
    A._check(lib.asd_csr_to_dia(n, A._p(xadj, C.c_uint32), A._p(adjncy, C.c_uint32), A._p(val9, C.c_double), ncomp,
                                None, None, C.byref(nd)))
    off = np.zeros(nd.value, dtype=np.int32)
    data = np.zeros((ncomp, nd.value, n), dtype=np.float64)
    A._check(lib.asd_csr_to_dia(n, A._p(xadj, C.c_uint32), A._p(adjncy, C.c_uint32), A._p(val9, C.c_double), ncomp,
                                A._p(off, C.c_int32), A._p(data, C.c_double), C.byref(nd)))
    return off, data


def dipole_nr(dim, nk=(1, 1, 1), abc=(3e-10, 3e-10, 3e-10), mu_scale=1.0, out=None):
    lib = A.load_library()
    dim, nk = _u32(dim), _u32(nk)
    abc = np.ascontiguousarray(abc, dtype=np.float64)
    mesh = [2 * int(d) * int(k) for d, k in zip(dim, nk)]
    P = int(np.prod(mesh))
    nr = np.zeros((9, P), dtype=np.float64) if out is None else out
    A._check(lib.asd_build_dipole_nr(A._p(dim, C.c_uint32), A._p(nk, C.c_uint32), A._p(abc, C.c_double), A.MUB,
                                     mu_scale, A._p(nr, C.c_double)))
    return nr, mesh


def fold_exchange(mesh, shell_vecs, J9, mu_muB, nr):
    lib = A.load_library()
    mesh = _u32(mesh)
    sv = np.ascontiguousarray(shell_vecs, dtype=np.int32).reshape(-1)
    j9 = np.ascontiguousarray(J9, dtype=np.float64).reshape(-1)
    cnt = C.c_uint32()
    A._check(lib.asd_fold_exchange_nr(A._p(mesh, C.c_uint32), len(sv) // 3, A._p(sv, C.c_int32),
                                      A._p(j9, C.c_double), mu_muB, A._p(nr, C.c_double), C.byref(cnt)))
    return cnt.value


def sc_mesh_xyz(dim):
    i, j, k = np.meshgrid(np.arange(dim[0]), np.arange(dim[1]), np.arange(dim[2]), indexing="ij")
    return np.stack([i.ravel(), j.ravel(), k.ravel()], axis=1).astype(np.uint32)


def _iso(J):
    return np.diag([J, J, J]).reshape(9)


SC_NN = [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]
SC_NNN = [(a, b, 0) for a in (1, -1) for b in (1, -1)] + [(a, 0, b) for a in (1, -1) for b in (1, -1)] + \
         [(0, a, b) for a in (1, -1) for b in (1, -1)]


def sc_ferromagnet(L, J=J_SC, mu=MU_SC, lam=0.1, k1u=K1U_SC, pbc=(1, 1, 1), T=0.0, J2=None, exch="csr",
                   dipole=False, abc=3e-10, stream=0):
    """Simple-cubic ferromagnet, spins ordered (i,j,k) with k innermost."""
    L = tuple(int(x) for x in (L if hasattr(L, "__len__") else (L, L, L)))
    vecs = list(SC_NN) + (list(SC_NNN) if J2 is not None else [])
    Js = [_iso(J)] * len(SC_NN) + ([_iso(J2)] * len(SC_NNN) if J2 is not None else [])
    nb = len(vecs)
    xadj, adj, val = build_csr(L, pbc, [mu], [0] * nb, [0] * nb, vecs, Js)
    n = L[0] * L[1] * L[2]
    s = A.SpinSystem(nspins=n, materials=[A.MaterialSpec(mu=mu, lam=lam, k1u=k1u, k1u_dir=(0, 0, 1))],
                     temperature=T, stream=stream)
    if exch == "csr":
        s.exch, s.xadj, s.adjncy, s.csr_val = A.EXCH_CSR, xadj, adj, val
    elif exch == "dia":
        off, data = csr_to_dia(n, xadj, adj, val, ncomp=3)
        s.exch, s.dia_offset, s.dia_val = A.EXCH_DIA, off, data
    s.meta = {"dim": L, "pbc": tuple(pbc), "nnz": len(adj), "kind": "sc"}
    if dipole:
        nr, mesh = dipole_nr(L, abc=(abc, abc, abc))
        s.lr, s.mesh, s.mesh_xyz, s.nr = A.LR_DIPOLE, mesh, sc_mesh_xyz(L), nr
    return s


def sc_fft(L, J=J_SC, mu=MU_SC, lam=0.1, k1u=K1U_SC, abc=3e-10, T=0.0):
    """sc, open boundaries; dipole (x mu) and NN exchange folded into one N_r (exchange method fft)."""
    L = tuple(int(x) for x in (L if hasattr(L, "__len__") else (L, L, L)))
    nr, mesh = dipole_nr(L, abc=(abc, abc, abc), mu_scale=mu)
    fold_exchange(mesh, [(1, 0, 0)], [_iso(J)], mu * A.MUB, nr)
    n = L[0] * L[1] * L[2]
    s = A.SpinSystem(nspins=n, materials=[A.MaterialSpec(mu=mu, lam=lam, k1u=k1u)], exch=A.EXCH_FFT, lr=A.LR_FFT,
                     mesh=mesh, mesh_xyz=sc_mesh_xyz(L), nr=nr, temperature=T)
    s.meta = {"dim": L, "kind": "sc_fft"}
    return s


# BCT-2: atom 0 at the cell corner, atom 1 at the body centre.  Shell 1: 8 body
# diagonals (other sublattice); shell 2: +-c; shell 3: 4 in-plane +-a; shell 4:
# 12 in-plane and out-of-plane face diagonals.  26 neighbours per site.
def _bct2_bonds(rng):
    shells = []
    diag_vecs = [(a, b, c) for a in (0, -1) for b in (0, -1) for c in (0, -1)]   # atom0 -> atom1 cells
    same2 = [(0, 0, 1), (0, 0, -1)]
    same3 = [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0)]
    same4 = [(a, b, 0) for a in (1, -1) for b in (1, -1)] + [(a, 0, b) for a in (1, -1) for b in (1, -1)] + \
            [(0, a, b) for a in (1, -1) for b in (1, -1)]
    tens = {}
    for key in [(0, 1, 1), (0, 0, 2), (1, 1, 2), (0, 0, 3), (1, 1, 3), (0, 0, 4), (1, 1, 4)]:
        d = rng.uniform(-2e-21, 1e-21, 3)
        D = rng.uniform(-1.0, 1.0, 3) * 0.05 * np.abs(d).mean()
        Jm = np.diag(d) + np.array([[0, D[2], -D[1]], [-D[2], 0, D[0]], [D[1], -D[0], 0]])
        tens[key] = Jm
    ba, bt, bv, bj = [], [], [], []
    for v in diag_vecs:                                 # 0 -> 1 with J, 1 -> 0 with J^T
        ba.append(0); bt.append(1); bv.append(v); bj.append(tens[(0, 1, 1)].reshape(9))
    for v in diag_vecs:
        ba.append(1); bt.append(0); bv.append(tuple(-x for x in v)); bj.append(tens[(0, 1, 1)].T.reshape(9))
    for sh, vecs in ((2, same2), (3, same3), (4, same4)):
        for a in (0, 1):
            Jm = tens[(a, a, sh)]
            for v in vecs:
                pos = v > (0, 0, 0)
                ba.append(a); bt.append(a); bv.append(v); bj.append((Jm if pos else Jm.T).reshape(9))
    return ba, bt, bv, bj


def bct2_antiferromagnet(L, layout="csr", mu=1.5, lam=0.01, k1u=-1e-23, T=0.0, seed=2):
    """BCT 2-sublattice antiferromagnet with easy-plane (hard-axis z) anisotropy."""
    L = tuple(int(x) for x in (L if hasattr(L, "__len__") else (L, L, L)))
    rng = np.random.default_rng(seed)
    ba, bt, bv, bj = _bct2_bonds(rng)
    xadj, adj, val = build_csr(L, (1, 1, 1), [mu, mu], ba, bt, bv, bj)
    n = 2 * L[0] * L[1] * L[2]
    mats = [A.MaterialSpec(mu=mu, lam=lam, k1u=k1u, k1u_dir=(0, 0, 1), sublattice=0),
            A.MaterialSpec(mu=mu, lam=lam, k1u=k1u, k1u_dir=(0, 0, 1), sublattice=1)]
    s = A.SpinSystem(nspins=n, materials=mats, full=True, temperature=T)
    if layout == "csr":
        s.exch, s.xadj, s.adjncy, s.csr_val = A.EXCH_CSR, xadj, adj, val
    else:
        off, data = csr_to_dia(n, xadj, adj, val)
        s.exch, s.dia_offset, s.dia_val = A.EXCH_DIA, off, data
    s.meta = {"dim": L, "nnz": len(adj), "kind": "bct2", "layout": layout}
    return s


def film_dia(Lx, Ly, Lz, J1=1e-21, J2=-2e-22, mu=MU_SC, lam=1e-4, k1u=0.0, dipole=True, abc=3e-10,
             pulse_width_sites=16.0):
    """Thin film, periodic in-plane, open along z; J1+J2 in DIA; optional dipole; sinc-in-space pulse profile."""
    L = (int(Lx), int(Ly), int(Lz))
    vecs = list(SC_NN) + list(SC_NNN)
    Js = [_iso(J1)] * 6 + [_iso(J2)] * 12
    xadj, adj, val = build_csr(L, (1, 1, 0), [mu], [0] * 18, [0] * 18, vecs, Js)
    n = L[0] * L[1] * L[2]
    off, data = csr_to_dia(n, xadj, adj, val, ncomp=3)
    s = A.SpinSystem(nspins=n, materials=[A.MaterialSpec(mu=mu, lam=lam, k1u=k1u)], exch=A.EXCH_DIA,
                     dia_offset=off, dia_val=data)
    xyz = sc_mesh_xyz(L).astype(np.float64)
    x = (xyz[:, 0] - L[0] / 2) / pulse_width_sites
    prof = np.zeros((n, 3))
    prof[:, 0] = np.sinc(x)                     # unit-amplitude profile; the amplitude is the ramp value
    s.site_field = prof
    s.meta = {"dim": L, "nnz": len(adj), "ndiag": len(off), "kind": "film"}
    if dipole:
        nr, mesh = dipole_nr(L, abc=(abc, abc, abc))
        s.lr, s.mesh, s.mesh_xyz, s.nr = A.LR_DIPOLE, mesh, sc_mesh_xyz(L), nr
    return s


def replica_batch(nrep=96, edges=(16, 24, 32, 48, 64), seed=4, Tmax=None, Tc=None):
    """Uneven sc replicas (config-0 material), edges drawn uniformly, temperatures 0..Tmax."""
    rng = np.random.default_rng(seed)
    L = rng.choice(np.asarray(edges), size=nrep)
    if Tmax is None:
        Tmax = 1.2 * (Tc if Tc is not None else 104.0)
    Ts = np.linspace(0.0, Tmax, nrep)
    reps = [sc_ferromagnet(int(l), T=float(t), stream=r) for r, (l, t) in enumerate(zip(L, Ts))]
    return reps, L, Ts


def pulse_amplitude(t_s, amp=0.1, t0=2e-13, sigma=5e-14):
    """Gaussian-in-time envelope of the site-field pulse [T]."""
    return amp * math.exp(-0.5 * ((t_s - t0) / sigma) ** 2)


def from_reference_inputs(ucf_path, exch_path, dim, pbc=(1, 1, 1), full=True, T=0.0, mesh_points=False):
    """A SpinSystem from the reference's own input files: the unit-cell file (.ucf) and the
    exchange file (.exch, unitcell method), on dim[0] x dim[1] x dim[2] cells.  Species and atoms
    coincide as in the unitcell exchange method (src/exch_unitcell.cpp:296-401).  Returns the
    system and the per-atom records (initial spins, positions)."""
    nms, atoms = A.read_ucf(ucf_path, mesh_points)
    if nms != len(atoms):
        raise ValueError("the unitcell exchange method pairs species with unit-cell atoms: nms must equal nauc")
    s1, s2, vec, J = A.read_exch(exch_path, nms)
    mus = [a["mu"] for a in atoms]
    xadj, adj, val = build_csr(dim, pbc, mus, s1, s2, vec, J.reshape(-1, 9))
    mats = [A.MaterialSpec(mu=a["mu"], lam=a["damping"], gamma=a["gamma"], k1u=a["k1u"], k1u_dir=a["k1u_dir"],
                           sublattice=a["sublattice"]) for a in atoms]
    n = int(np.prod(dim)) * len(atoms)
    s = A.SpinSystem(nspins=n, materials=mats, full=full, temperature=T, exch=A.EXCH_CSR, xadj=xadj, adjncy=adj,
                     csr_val=val)
    s.meta = {"dim": tuple(dim), "nnz": len(adj), "kind": "reference-inputs"}
    return s, atoms
