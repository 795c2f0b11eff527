"""Shared test helpers: rebuild systems from golden fixtures, run product and oracle side by side."""
import os

import numpy as np

import asd_b200 as A

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def system_from_npz(d):
    mats = [A.MaterialSpec(mu=m[0], lam=m[1], gamma=m[2], k1u=m[3], k1u_dir=tuple(m[4:7]), sublattice=int(m[7]))
            for m in d["mat"]]
    s = A.SpinSystem(nspins=int(d["nspins"]), materials=mats, exch=int(d["exch"]), full=bool(d["full"]),
                     temperature=float(d["T"]))
    if s.exch == A.EXCH_CSR:
        s.xadj, s.adjncy, s.csr_val = d["xadj"], d["adjncy"], d["csr_val"]
    if s.exch == A.EXCH_DIA:
        s.dia_offset, s.dia_val = d["dia_offset"], d["dia_val"]
    return s


def load(name):
    return np.load(os.path.join(GOLDEN, name))


def maxdiff(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max())


def plaquette_quartets(L):
    """For every spin of an L^3 periodic sc lattice, the (j, k, l) of the four xy plaquettes it
    belongs to, ordered around the plaquette."""
    idx = lambda x, y, z: ((x % L) * L + (y % L)) * L + (z % L)
    xadj, J, K, Lq = [0], [], [], []
    for x in range(L):
        for y in range(L):
            for z in range(L):
                for dx, dy in ((1, 1), (-1, 1), (-1, -1), (1, -1)):
                    J.append(idx(x + dx, y, z)); K.append(idx(x + dx, y + dy, z)); Lq.append(idx(x, y + dy, z))
                xadj.append(len(J))
    return [np.array(a, dtype=np.uint32) for a in (xadj, J, K, Lq)]
