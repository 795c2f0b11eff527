"""FP64 CPU restatement of the Heun step with the long-range field evaluated by FFT.

TEST INFRASTRUCTURE ONLY: imported by tests/ and by bench.py's CPU legs (the reference arm and
`cpu_baseline`), never by the product.  It loads no library of the product: lattices come from
the numpy builders below and the dipole matrix from liboracle.so (the C restatement).

Why it exists.  The reference evaluates the dipole field by FFT (GPU: src/cufields.cu:248-462 with
src/cuda_util.cu:76,97,245,250; CPU: FFTW in src/fields.cpp:253-339, which cannot be built here:
FFTW3 is absent).  The direct-sum oracle (asd_oracle.c `longrange_field`) evaluates the same cyclic
convolution in O(N^2) and is limited to a few thousand spins; this restatement evaluates it with
scipy's pocketfft (threaded, FP64) so that a 1M-spin lattice runs on the host cores.  It is pinned
against the direct-sum oracle on small lattices (tests/test_fft_oracle.py).

Semantics (default flags of the oracle: the reference CUDA path with its bugs fixed):
  * Heun, src/cuint.cu:60-242 (CHeun1/CHeun2): H = HDemag + sum_j J_ij S_j + H_app + site field
    + K1u (S.n) n; f = llgpf (S x H + lambda S x (S x H)), llgpf = -1/(1+lambda^2);
    S' = (S + rdt f(S)) / |.|;  S_n+1 = (S + rdt (f(S) + f(S'))/2) / |.|, rdt = dt * 1.76e11.
  * ASD_LR_DIPOLE: HDemag = IFFT(N_k FFT(mu S)) / P at the spin sites, from S at the first stage
    of every `update`-th step and kept for both stages (src/cuda.cu:47-90).
  * ASD_LR_FFT: the whole field of each stage from the interaction matrix (exchange folded in,
    src/cuda.cu:101-112).
  * T = 0 only (no thermal term); the 1M-spin dipole lattice it times is a T = 0 workload.

The transform is pruned to the spins' bounding box as the device path is: a real FFT along z of
the box rows, complex FFTs along y then x of the rows that hold data, the 3x3 product with N_k on
the half spectrum, and the inverse passes producing only the box.  The cyclic convolution depends
only on mesh differences, so the box is shifted to the mesh origin first.
"""
from __future__ import annotations

import ctypes as C
import os
import time
from types import SimpleNamespace

import numpy as np
import scipy.fft as sfft
import scipy.sparse as sp

from . import oracle as O

MUB, GYRO = O.MUB, O.GYRO
SC_NN = [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def sc_csr(L, J, mu, pbc=(0, 0, 0), vecs=SC_NN):
    """CSR of a simple-cubic lattice with isotropic bonds `vecs`, rows in spin order (i, j, k) with
    k innermost and each row's entries in bond order, out-of-range bonds dropped on open axes and
    wrapped on periodic ones: the rows exch::exchunitcell builds for one species
    (src/exch_unitcell.cpp:296-401; bit-exact against it in tests/test_fft_oracle.py).
    Values J/(mu muB) [T] on the diagonal; returns xadj, adjncy, val (nnz x 9)."""
    L = np.asarray(L, dtype=np.int64)
    n = int(np.prod(L))
    idx = np.arange(n, dtype=np.int64)
    xyz = np.stack([idx // (L[1] * L[2]), (idx // L[2]) % L[1], idx % L[2]], axis=1)
    cols, ok = [], []
    for v in vecs:
        q = xyz + np.asarray(v, dtype=np.int64)
        good = np.ones(n, dtype=bool)
        for a in range(3):
            if pbc[a]:
                q[:, a] %= L[a]
            else:
                good &= (q[:, a] >= 0) & (q[:, a] < L[a])
        cols.append((q[:, 0] * L[1] + q[:, 1]) * L[2] + q[:, 2])
        ok.append(good)
    cols = np.stack(cols, axis=1)
    ok = np.stack(ok, axis=1)
    counts = ok.sum(1)
    xadj = np.zeros(n + 1, dtype=np.uint32)
    xadj[1:] = np.cumsum(counts)
    adj = cols[ok].astype(np.uint32)             # row-major: each row's bonds in bond order
    val = np.zeros((len(adj), 9))
    v = J / (mu * MUB)
    val[:, 0] = val[:, 4] = val[:, 8] = v
    return xadj, adj, val


def sc_mesh_xyz(L):
    i, j, k = np.meshgrid(np.arange(L[0]), np.arange(L[1]), np.arange(L[2]), indexing="ij")
    return np.stack([i.ravel(), j.ravel(), k.ravel()], axis=1).astype(np.uint32)


def dipole_nr(L, abc=3e-10, mu_scale=1.0):
    """Real-space point-dipole matrix [9][P] on the 2L mesh: intmat::fillDipIntmat
    (src/intmat.cpp:263-331) as restated in asd_oracle.c `orc_build_dipole_nr`."""
    lib = O.olib()
    dim = O.au32(L)
    nk = O.au32([1, 1, 1])
    a = O.a64([abc, abc, abc])
    mesh = [2 * int(x) for x in L]
    nr = np.zeros((9, int(np.prod(mesh))))
    lib.orc_build_dipole_nr(O._ptr(dim, C.c_uint32), O._ptr(nk, C.c_uint32), O._ptr(a, C.c_double), MUB, mu_scale,
                            O._ptr(nr, C.c_double))
    return nr, mesh


def sc_dipole_system(L, J=1e-21, mu=1.5, lam=0.1, k1u=1e-23, pbc=(0, 0, 0), abc=3e-10):
    """The simple-cubic ferromagnet with CSR nearest-neighbour exchange and the point-dipole field
    (the 1M-spin dipole lattice at L = (128, 128, 64), open boundaries), as a plain record."""
    L = tuple(int(x) for x in L)
    xadj, adj, val = sc_csr(L, J, mu, pbc)
    nr, mesh = dipole_nr(L, abc)
    mat = SimpleNamespace(mu=mu, lam=lam, gamma=1.0, k1u=k1u, k1u_dir=(0.0, 0.0, 1.0), sublattice=0)
    return SimpleNamespace(nspins=int(np.prod(L)), materials=[mat], atom=None, exch=O.EXCH_CSR, full=False,
                           xadj=xadj, adjncy=adj, csr_val=val, lr=O.LR_DIPOLE, mesh=mesh, mesh_xyz=sc_mesh_xyz(L),
                           nr=nr, temperature=0.0, stream=0, site_field=None, meta={"dim": L})


def random_spins(n, seed):
    """The bench's initial spins: z ~ U[-1,1), phi ~ U[0,2pi) from numpy PCG64(seed)."""
    rng = np.random.default_rng(seed)
    z = rng.uniform(-1.0, 1.0, n)
    phi = rng.uniform(0.0, 2.0 * np.pi, n)
    r = np.sqrt(1.0 - z * z)
    return np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=1)


class FFTOracle:
    """FP64 Heun step of one lattice (CSR/DIA-free exchange in CSR form, long-range by FFT)."""

    def __init__(self, system, dt=1e-16, applied=(0.0, 0.0, 0.0), update=1, workers=None):
        s = system
        if s.temperature != 0.0:
            raise NotImplementedError("the FFT restatement runs T = 0 only")
        self.n = n = int(s.nspins)
        self.workers = workers or host_threads()
        nm = len(s.materials)
        atoms = np.asarray(s.atom) if s.atom is not None else np.arange(n) % nm
        self.llgpf = np.empty(n)
        self.lam = np.empty(n)
        self.k1u = np.empty(n)
        self.k1d = np.empty((n, 3))
        w = np.empty(n)
        for t, m in enumerate(s.materials):
            sel = atoms == t
            self.llgpf[sel] = -1.0 / (1.0 + m.lam * m.lam)        # src/llg.cpp:629
            self.lam[sel] = m.lam
            self.k1u[sel] = 2.0 * m.k1u / (MUB * m.mu)          # src/llg.cpp:591-592
            self.k1d[sel] = m.k1u_dir
            w[sel] = m.mu
        self.rdt = dt * GYRO
        self.applied = np.asarray(applied, dtype=np.float64)
        self.update = max(int(update), 1)
        self.site = None if s.site_field is None else np.asarray(s.site_field, dtype=np.float64).reshape(n, 3)
        self.exch = None
        if s.exch == O.EXCH_CSR:
            xadj = np.asarray(s.xadj, dtype=np.int64)
            adj = np.asarray(s.adjncy, dtype=np.int64)
            val = np.asarray(s.csr_val, dtype=np.float64).reshape(-1, 9)
            comps = range(9) if s.full else (0, 4, 8)
            self.full = bool(s.full)
            self.exch = {q: sp.csr_matrix((val[:, q], adj, xadj), shape=(n, n)) for q in comps}
        self.lr = int(s.lr or 0)
        if self.lr:
            self._setup_lr(s, w)
        self.S = np.zeros((n, 3))
        self.hd = np.zeros((n, 3))
        self.t = 0

    # ---------------------------------------------------------------- long-range field
    def _setup_lr(self, s, w):
        mesh = [int(x) for x in s.mesh]
        xyz = np.asarray(s.mesh_xyz, dtype=np.int64).reshape(-1, 3)
        lo = xyz.min(0)
        hi = xyz.max(0)
        self.mesh = mesh
        self.box = [int(x) for x in (hi - lo + 1)]
        self.pos = tuple((xyz - lo).T)                         # box-local positions
        self.w = w if self.lr == O.LR_DIPOLE else np.ones(self.n)
        nr = np.asarray(s.nr, dtype=np.float64).reshape(9, *mesh)
        sym = all(np.array_equal(nr[a], nr[b]) for a, b in ((1, 3), (2, 6), (5, 7)))
        comps = (0, 1, 2, 4, 5, 8) if sym else tuple(range(9))
        nk = {}
        for q in comps:
            k = sfft.rfftn(nr[q], workers=self.workers)
            nk[q] = k.real.copy() if np.abs(k.imag).max() <= 1e-12 * max(np.abs(k.real).max(), 1e-300) else k
        if sym:
            nk[3], nk[6], nk[7] = nk[1], nk[2], nk[5]
        self.nk = nk

    def lr_field(self, S):
        """IFFT(N_k FFT(w S)) / P at the spin sites (pruned to the spins' box)."""
        m0, m1, m2 = self.mesh
        bx, by, bz = self.box
        W = self.workers
        M = np.zeros((3, bx, by, m2))
        ws = S * self.w[:, None]
        for c in range(3):
            M[c][self.pos] = ws[:, c]
        Z = sfft.rfft(M, axis=3, workers=W)                   # (3, bx, by, m2/2+1)
        del M
        Y = sfft.fft(Z, n=m1, axis=2, workers=W)               # (3, bx, m1, kz)
        del Z
        X = sfft.fft(Y, n=m0, axis=1, workers=W)               # (3, m0, m1, kz)
        del Y
        nk = self.nk
        H = np.empty_like(X)
        for a in range(3):
            H[a] = nk[3 * a] * X[0] + nk[3 * a + 1] * X[1] + nk[3 * a + 2] * X[2]
        del X
        Y2 = sfft.ifft(H, axis=1, workers=W)[:, :bx]
        del H
        Z2 = sfft.ifft(Y2, axis=2, workers=W)[:, :, :by]
        del Y2
        R = sfft.irfft(Z2, n=m2, axis=3, workers=W)
        out = np.empty((self.n, 3))
        for c in range(3):
            out[:, c] = R[c][self.pos]
        return out

    # ---------------------------------------------------------------- step
    def _exch(self, S):
        h = np.zeros((self.n, 3))
        if self.exch is None:
            return h
        if self.full:
            for a in range(3):
                for b in range(3):
                    h[:, a] += self.exch[3 * a + b] @ S[:, b]
        else:
            for a in range(3):
                h[:, a] = self.exch[4 * a] @ S[:, a]
        return h

    def _stage_field(self, S):
        if self.lr == O.LR_FFT:
            return self.lr_field(S)
        return self.hd + self._exch(S)

    def _rhs(self, S, h):
        H = h + self.applied
        if self.site is not None:
            H = H + self.site
        sn = np.einsum("ij,ij->i", S, self.k1d)
        H = H + (self.k1u * sn)[:, None] * self.k1d
        a = np.cross(S, H)
        b = np.cross(S, a)
        return self.llgpf[:, None] * (a + self.lam[:, None] * b)

    def set_spins(self, S):
        S = np.asarray(S, dtype=np.float64).reshape(self.n, 3)
        self.S = S / np.sqrt(np.einsum("ij,ij->i", S, S))[:, None]

    def spins(self):
        return self.S.copy()

    def field(self):
        """Exchange + long-range field of the current spins (no anisotropy, applied or site term)."""
        if self.lr == O.LR_DIPOLE:
            return self.lr_field(self.S) + self._exch(self.S)
        return self._stage_field(self.S)

    def step(self, k=1):
        for _ in range(int(k)):
            S = self.S
            if self.lr == O.LR_DIPOLE and self.t % self.update == 0:
                self.hd = self.lr_field(S)
            f1 = self._rhs(S, self._stage_field(S))
            es = S + f1 * self.rdt
            es /= np.sqrt(np.einsum("ij,ij->i", es, es))[:, None]
            f2 = self._rhs(es, self._stage_field(es))
            ps = S + 0.5 * (f1 + f2) * self.rdt
            self.S = ps / np.sqrt(np.einsum("ij,ij->i", ps, ps))[:, None]
            self.t += 1

    def timed_steps(self, k):
        """Wall time of k steps [s] (the spins are advanced)."""
        t0 = time.perf_counter()
        self.step(k)
        return time.perf_counter() - t0
