"""C-ABI boundary on the CPU: the library loads, exports every entry point the
header declares, and its host-side set-up builders agree with the oracle's
restatements of the reference set-up code."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import asd_b200 as A
import asd_lattice as LT
from conftest import REPO, has_gpu
from oracle import oracle as O

HEADER = os.path.join(REPO, "include", "asd.h")


def declared():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(asd_\w+)\s*\(", txt, flags=re.M)))


def test_library_exports_every_declared_symbol():
    lib = A.load_library()
    names = declared()
    assert len(names) >= 25
    out = subprocess.run(["nm", "-D", "--defined-only", A.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (asd_\w+)", out))
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    for n in names:
        getattr(lib, n)
    assert set(A.EXPORTED) <= set(names)


def test_version_string():
    assert "sm_100a" in A.version()


@pytest.mark.skipif(has_gpu(), reason="checks the no-device error path")
def test_create_without_device_fails_loudly():
    s = LT.sc_ferromagnet(4)
    with pytest.raises(A.AsdError) as e:
        A.Handle(A.RunParams(), s)
    assert e.value.code == A.ASD_ECUDA


def brute_sc_csr(L, pbc):
    n = L ** 3
    rows = []
    for i in range(L):
        for j in range(L):
            for k in range(L):
                nb = []
                for v in LT.SC_NN:
                    c = [i + v[0], j + v[1], k + v[2]]
                    ok = True
                    for x in range(3):
                        if c[x] < 0 or c[x] >= L:
                            if not pbc[x]:
                                ok = False
                            c[x] %= L
                    if ok:
                        nb.append((c[0] * L + c[1]) * L + c[2])
                rows.append(nb)
    return rows


@pytest.mark.parametrize("pbc", [(1, 1, 1), (1, 1, 0), (0, 0, 0)])
def test_build_csr_matches_neighbour_enumeration(pbc):
    L = 5
    s = LT.sc_ferromagnet(L, pbc=pbc)
    rows = brute_sc_csr(L, pbc)
    assert s.xadj[-1] == sum(len(r) for r in rows)
    for i, r in enumerate(rows):
        assert list(s.adjncy[s.xadj[i]:s.xadj[i + 1]]) == r
    assert np.allclose(s.csr_val[:, 0], LT.J_SC / (LT.MU_SC * A.MUB), rtol=0, atol=0)
    assert np.all(s.csr_val[:, [1, 2, 3, 5, 6, 7]] == 0)


def test_bct2_hermitian_pairs():
    s = LT.bct2_antiferromagnet(3)
    n = s.nspins
    assert np.all(np.diff(s.xadj) == 26)
    M = {}
    for i in range(n):
        for k in range(s.xadj[i], s.xadj[i + 1]):
            M[(i, int(s.adjncy[k]))] = s.csr_val[k].reshape(3, 3)
    for (i, j), m in M.items():
        assert np.array_equal(M[(j, i)], m.T)


def test_csr_to_dia_keeps_the_last_diagonal_the_reference_drops():
    # BCT-2 with periodic wrap always couples spin 0 to spin N-1 (offset N-1); the reference's
    # scan (src/matrix_conv.cpp:43) skips that diagonal, the product keeps it.
    s = LT.bct2_antiferromagnet(3)
    n = s.nspins
    off, data = LT.csr_to_dia(n, s.xadj, s.adjncy, s.csr_val)
    assert off[-1] == n - 1
    xadj, adj, val = O.au32(s.xadj), O.au32(s.adjncy), O.a64(s.csr_val)
    nd = O.olib().orc_csr_to_dia(n, O._ptr(xadj, C.c_uint32), O._ptr(adj, C.c_uint32), O._ptr(val, C.c_double), None, None)
    assert nd == len(off) - 1


def test_csr_to_dia_matches_oracle_restatement():
    for s in [LT.sc_ferromagnet(5), LT.sc_ferromagnet(4, pbc=(1, 0, 1)), LT.sc_ferromagnet(6, J2=-2e-22)]:
        n = s.nspins
        off, data = LT.csr_to_dia(n, s.xadj, s.adjncy, s.csr_val)
        L = O.olib()
        xadj, adj, val = O.au32(s.xadj), O.au32(s.adjncy), O.a64(s.csr_val)
        nd = L.orc_csr_to_dia(n, O._ptr(xadj, C.c_uint32), O._ptr(adj, C.c_uint32), O._ptr(val, C.c_double), None, None)
        off2 = np.zeros(nd, dtype=np.int32)
        data2 = np.zeros((9, nd, n))
        L.orc_csr_to_dia(n, O._ptr(xadj, C.c_uint32), O._ptr(adj, C.c_uint32), O._ptr(val, C.c_double),
                         O._ptr(off2, C.c_int32), O._ptr(data2, C.c_double))
        assert np.array_equal(off, off2) and np.array_equal(data, data2)
        off3, data3 = LT.csr_to_dia(n, s.xadj, s.adjncy, s.csr_val, ncomp=3)
        assert np.array_equal(off3, off2) and np.array_equal(data3, data2[[0, 4, 8]])


def test_dipole_nr_matches_oracle_restatement():
    dim, nk, abc = np.array([3, 4, 2], np.uint32), np.array([1, 1, 1], np.uint32), np.array([3e-10, 3e-10, 4e-10])
    nr, mesh = LT.dipole_nr(dim, nk, abc, mu_scale=1.5)
    nr2 = np.zeros_like(nr)
    O.olib().orc_build_dipole_nr(O._ptr(dim, C.c_uint32), O._ptr(nk, C.c_uint32), O._ptr(abc, C.c_double), A.MUB, 1.5,
                                 O._ptr(nr2, C.c_double))
    assert np.allclose(nr, nr2, rtol=1e-15, atol=0)
    # point-dipole tensor is symmetric and traceless away from the origin
    P = nr.shape[1]
    t = nr[0] + nr[4] + nr[8]
    assert np.abs(t).max() < 1e-12 * np.abs(nr).max()
    for a, b in ((1, 3), (2, 6), (5, 7)):   # symmetric up to the rounding of (3 e_a) e_b
        assert np.allclose(nr[a], nr[b], rtol=1e-15, atol=1e-30)


def test_fold_exchange_matches_oracle_restatement():
    mesh = np.array([8, 8, 8], np.uint32)
    J9 = np.diag([1e-21, 1e-21, 1e-21]).reshape(1, 9)
    nr = np.zeros((9, 512))
    cnt = LT.fold_exchange(mesh, [(1, 0, 0)], J9, 1.5 * A.MUB, nr)
    assert cnt == 6
    nr2 = np.zeros_like(nr)
    sv = np.array([1, 0, 0], np.int32)
    c2 = O.olib().orc_fold_exchange_nr(O._ptr(mesh, C.c_uint32), 1, O._ptr(sv, C.c_int32), O._ptr(O.a64(J9), C.c_double),
                                       1.5 * A.MUB, O._ptr(nr2, C.c_double))
    assert c2 == 6 and np.array_equal(nr, nr2)
    cnt = LT.fold_exchange(mesh, [(1, 1, 0)], J9, 1.5 * A.MUB, np.zeros((9, 512)))
    assert cnt == 12


def test_builder_rejects_bad_input():
    lib = A.load_library()
    nnz = C.c_uint32()
    assert lib.asd_build_csr(None, None, 0, None, 0, None, None, None, None, 0.0, None, None, None, C.byref(nnz)) == A.ASD_EINVAL
    xadj = np.array([0, 1], np.uint32)
    adj = np.array([5], np.uint32)  # out of range
    nd = C.c_uint32()
    assert lib.asd_csr_to_dia(1, A._p(xadj, C.c_uint32), A._p(adj, C.c_uint32), None, 9, None, None, C.byref(nd)) == A.ASD_EINVAL
