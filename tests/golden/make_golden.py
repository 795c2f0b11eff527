"""Generate the golden vectors in this directory from the reference itself.

Runs the reference's own llgCPU::llgCPU (src/llgCPU.cpp) compiled from the
reference sources by oracle/Makefile (oracle/_ref/libref_llgcpu*.so) on small
seeded inputs and stores inputs + outputs as .npz.  Needs the reference tree
(it is not present where the tests run later); run from the repository root:
    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [REPO, os.path.join(REPO, "gpu-atomistic-code_b200"), os.path.dirname(HERE)]

import asd_lattice as LT  # noqa: E402
from oracle import oracle as O  # noqa: E402
from helpers import plaquette_quartets  # noqa: E402


def save(name, s, S0, out, **extra):
    d = dict(S0=S0, out=out, nspins=s.nspins, exch=s.exch, full=int(s.full), T=s.temperature,
             mat=np.array([[m.mu, m.lam, m.gamma, m.k1u, *m.k1u_dir, m.sublattice] for m in s.materials]))
    if s.exch == 2:
        d.update(xadj=s.xadj, adjncy=s.adjncy, csr_val=s.csr_val)
    if s.exch == 1:
        d.update(dia_offset=s.dia_offset, dia_val=s.dia_val)
    d.update(extra)
    np.savez_compressed(os.path.join(HERE, name), **d)
    print(name, s.nspins, "spins", float(np.abs(out - S0).max()))


def main():
    O.build()
    s = LT.sc_ferromagnet(6)
    S0 = LT.random_spins(s.nspins, 0)
    r = O.RefLLGCPU(s); r.set_spins(S0); r.step(200)
    save("ref_sc6_csr_T0_200.npz", s, S0, r.spins(), steps=200)

    s = LT.sc_ferromagnet(6, T=300.0)
    r = O.RefLLGCPU(s, seed=(7, 107)); r.set_spins(S0); r.step(50)
    save("ref_sc6_csr_T300_mwc_50.npz", s, S0, r.spins(), steps=50, mwc=np.array([7, 107]))

    s = LT.bct2_antiferromagnet(3, layout="csr")
    S1 = LT.random_spins(s.nspins, 1)
    r = O.RefLLGCPU(s); r.set_spins(S1); r.step(100)
    save("ref_bct3_csr_full_T0_100.npz", s, S1, r.spins(), steps=100)

    s = LT.sc_ferromagnet(6, exch="dia")
    r = O.RefLLGCPU(s); r.set_spins(S0); r.step(100)
    save("ref_sc6_dia_T0_100.npz", s, S0, r.spins(), steps=100)

    s = LT.sc_ferromagnet(4, T=300.0, pbc=(1, 1, 0))
    S2 = LT.random_spins(s.nspins, 2)
    xi = np.concatenate([O.thermal_normals(5, 0, s.nspins, t).reshape(-1) for t in range(20)])
    r = O.RefLLGCPU(s, replay=True); r.set_noise(xi); r.set_spins(S2); r.step(20)
    save("ref_sc4_open_T300_replay_20.npz", s, S2, r.spins(), steps=20, noise=xi)
    four_spin_case()


def four_spin_case():
    """llgCPU with the four-spin term (src/llgCPU.cpp:142-170,275-297) on xy plaquettes, MWC noise."""
    s = LT.sc_ferromagnet(5, T=300.0)
    S0 = LT.random_spins(s.nspins, 3)
    q = plaquette_quartets(5)
    r = O.RefLLGCPU(s, seed=(7, 107)); r.set_four_spin(*q, 30.0); r.set_spins(S0); r.step(30)
    save("ref_sc5_fourspin_T300_mwc_30.npz", s, S0, r.spins(), steps=30, mwc=np.array([7, 107]),
         q4_xadj=q[0], q4_j=q[1], q4_k=q[2], q4_l=q[3], q4_jq=30.0)


if __name__ == "__main__":
    main()
