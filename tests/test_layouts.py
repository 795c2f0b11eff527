"""A CSR matrix whose entries lie on few diagonals (a regular lattice) also runs on the typed DIA
gather (columns formed from the row and the diagonal); the autotuner picks between the layouts.
On either layout the results stay within the parity tolerances of the oracle: FP32 1e-5, fused
FP64 1e-10 (the DIA gather sums a row in ascending diagonal order, the SELL gather in the CSR
order, so the two differ in rounding only)."""
import numpy as np
import pytest

import asd_b200 as A
import asd_lattice as LT
from helpers import maxdiff
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def run(s, precision, layout, steps=200, T=0.0, update=1):
    S0 = LT.random_spins(s.nspins, 0)
    flags = A.FLAG_COMPENSATED if precision == A.FP32 else 0
    with A.Handle(A.RunParams(precision=precision, flags=flags, update=update, seed=2), s) as h:
        h.set_device_layout(layout)
        h.set_spins(S0)
        h.step(steps)
        return h.get_spins()


@pytest.mark.parametrize("case", ["sc8_periodic", "sc2_periodic_duplicates", "film_open_z", "dipole_open"])
@pytest.mark.parametrize("precision,tol", [(A.FP32, 1e-5), (A.FP64_FUSED, 1e-10)])
def test_csr_matrix_on_dia_layout_matches_oracle(gpu, case, precision, tol):
    if case == "sc8_periodic":
        s = LT.sc_ferromagnet(8, T=0.0)
    elif case == "sc2_periodic_duplicates":          # +x and -x reach the same neighbour: summed
        s = LT.sc_ferromagnet(2)
    elif case == "film_open_z":
        s = LT.sc_ferromagnet((8, 6, 3), pbc=(1, 1, 0))
    else:
        s = LT.sc_ferromagnet((8, 8, 4), pbc=(0, 0, 0), dipole=True)
    o = O.Oracle(s, update=1)
    o.set_spins(LT.random_spins(s.nspins, 0))
    o.step(200)
    for layout in (A.EXCH_DIA, A.EXCH_CSR):
        g = run(s, precision, layout)
        assert maxdiff(g, o.spins()) <= tol, (layout, maxdiff(g, o.spins()))


def test_matrix_on_many_diagonals_has_no_dia_layout(gpu):
    s = LT.bct2_antiferromagnet(5)                   # periodic 26-neighbour shells: > 32 diagonals
    with A.Handle(A.RunParams(precision=A.FP32, flags=A.FLAG_COMPENSATED), s) as h:
        with pytest.raises(A.AsdError):
            h.set_device_layout(A.EXCH_DIA)


def test_autotuner_considers_both_layouts(gpu):
    s = LT.sc_ferromagnet((16, 16, 8), pbc=(0, 0, 0))
    with A.Handle(A.RunParams(precision=A.FP32, flags=A.FLAG_COMPENSATED | A.FLAG_AUTOTUNE), s) as h:
        t = h.tuning()
    assert "SELL:" in t and "DIA:" in t, t
