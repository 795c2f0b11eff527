"""asd_magnetisation against the per-(replica, sublattice) means of the spins computed on the
host, in every form: one replica (the last partial-sum block forms the means, one launch), two
sublattices, a few replicas (still one launch), many replicas (a separate reduction launch), and
calls repeated between steps (the block ticket rearms itself); into pageable and page-locked
host buffers."""
import numpy as np
import pytest

import asd_b200 as A
import asd_lattice as LT

pytestmark = pytest.mark.gpu


def host_means(systems, spins):
    out, off = [], 0
    nsub = max(max(m.sublattice for m in s.materials) for s in systems) + 1
    for s in systems:
        n = s.nspins
        atom = np.arange(n) % len(s.materials) if s.atom is None else np.asarray(s.atom)
        sub = np.array([s.materials[m].sublattice for m in atom])
        blk = spins[off:off + n]
        out.append([blk[sub == q].mean(axis=0) if np.any(sub == q) else np.zeros(3) for q in range(nsub)])
        off += n
    return np.array(out)


CASES = {
    "one replica, 24 chunks": lambda: [LT.sc_ferromagnet((40, 30, 20))],
    "two sublattices": lambda: [LT.bct2_antiferromagnet(12)],
    "4 replicas (12 means)": lambda: [LT.sc_ferromagnet(8 + k, stream=k) for k in range(4)],
    "20 replicas (60 means)": lambda: [LT.sc_ferromagnet(6 + k % 3, stream=k) for k in range(20)],
}


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("prec", [A.FP64_PLAIN, A.FP32, A.FP64_FUSED])
@pytest.mark.parametrize("buf", ["pageable", "page-locked"])
def test_magnetisation_matches_host_means(gpu, case, prec, buf):
    """A page-locked output buffer takes the means from the kernel itself (no copy): it is
    filled with NaN before every call, so a store that never came shows."""
    import torch

    systems = CASES[case]()
    n = sum(s.nspins for s in systems)
    flags = A.FLAG_COMPENSATED if prec == A.FP32 else 0
    with A.Handle(A.RunParams(precision=prec, flags=flags), systems) as h:
        h.set_spins(LT.random_spins(n, 9))
        nq = h.nrep * h.nsub * 3
        out = torch.empty(nq, dtype=torch.float64).pin_memory().numpy() if buf == "page-locked" else np.empty(nq)
        for _ in range(3):
            h.step(2)
            out[:] = np.nan
            got = h.magnetisation(out)
            want = host_means(systems, h.get_spins())
            assert got.shape == want.shape, (got.shape, want.shape)
            err = float(np.abs(got - want).max())
            assert err <= 1e-14, (case, prec, err)
