"""Set-up data: the library's CSR assembly and CSR->DIA conversion against the reference's own
exch::exchunitcell and matconv::csr_to_dia_* (compiled from source into oracle/_ref), and the
readers of the reference's input files (.ucf, .exch, csr_exch_mat.dat)."""
import os

import numpy as np
import pytest

import asd_b200 as A
import asd_lattice as LT
from oracle import oracle as O

HAVE_REF_BUILDERS = os.path.exists(O.REF_BUILDERS_SO) or os.path.isdir(os.path.join(O.reference_dir(), "src"))
needs_ref = pytest.mark.skipif(not HAVE_REF_BUILDERS, reason="reference builders not built")


def _sorted_bonds(ba, bt, bv, bj):
    """Bonds grouped by (atom, neighbour atom), shell order kept: the order exchunitcell visits."""
    order = sorted(range(len(ba)), key=lambda b: (ba[b], bt[b]))
    return ([ba[b] for b in order], [bt[b] for b in order], [bv[b] for b in order],
            [np.asarray(bj[b]).reshape(9) for b in order])


def _cases():
    rng = np.random.default_rng(2)
    sc = ([0] * 6, [0] * 6, list(LT.SC_NN), [LT._iso(1e-21)] * 6)
    bct = _sorted_bonds(*LT._bct2_bonds(rng))
    return [("sc", (5, 4, 3), [1.5], sc), ("bct2", (4, 3, 5), [1.5, 2.1], bct)]


@needs_ref
@pytest.mark.parametrize("pbc", [(1, 1, 1), (1, 0, 1), (0, 0, 0)])
@pytest.mark.parametrize("case", [0, 1])
def test_build_csr_matches_reference_exchunitcell(case, pbc):
    name, dim, mus, (ba, bt, bv, bj) = _cases()[case]
    xadj, adj, val = LT.build_csr(dim, pbc, mus, ba, bt, bv, bj)
    bonds = list(zip(ba, bt, bv, bj))
    rx, ra, rv = O.ref_exchunitcell(dim, pbc, mus, bonds, offdiag=True)
    assert np.array_equal(xadj, rx)
    assert np.array_equal(adj, ra)
    assert np.array_equal(val, rv)            # J/(mu muB): same expression, bit for bit
    rx2, ra2, rv2 = O.ref_exchunitcell(dim, pbc, mus, bonds, offdiag=False)
    assert np.array_equal(ra2, adj) and np.array_equal(rv2[:, [0, 4, 8]], val[:, [0, 4, 8]])


@needs_ref
@pytest.mark.parametrize("pbc", [(1, 1, 1), (0, 1, 0)])
def test_csr_to_dia_matches_reference_sc(pbc):
    name, dim, mus, (ba, bt, bv, bj) = _cases()[0]
    xadj, adj, val = LT.build_csr(dim, pbc, mus, ba, bt, bv, bj)
    n = len(xadj) - 1
    for ncomp, offdiag in ((3, False), (9, True)):
        off, data = LT.csr_to_dia(n, xadj, adj, val, ncomp=ncomp)
        roff, rdata = O.ref_csr_to_dia(n, xadj, adj, val, offdiag=offdiag)
        assert np.array_equal(off, roff)
        comps = [0, 4, 8] if ncomp == 3 else list(range(9))
        for c, q in enumerate(comps):
            assert np.array_equal(data[c].reshape(-1), rdata[q]), (ncomp, q)


@needs_ref
def test_csr_to_dia_bct2_differs_only_by_the_dropped_last_diagonal():
    """Periodic BCT-2 couples spin 0 and spin N-1 (offset N-1): the reference's diagonal scan
    stops at N-2 and loses that diagonal; every other diagonal is identical."""
    name, dim, mus, (ba, bt, bv, bj) = _cases()[1]
    xadj, adj, val = LT.build_csr(dim, (1, 1, 1), mus, ba, bt, bv, bj)
    n = len(xadj) - 1
    off, data = LT.csr_to_dia(n, xadj, adj, val, ncomp=9)
    roff, rdata = O.ref_csr_to_dia(n, xadj, adj, val, offdiag=True)
    assert n - 1 in set(off.tolist()) and n - 1 not in set(roff.tolist())
    keep = [k for k, o in enumerate(off) if o != n - 1]
    assert np.array_equal(off[keep], roff)
    for q in range(9):
        assert np.array_equal(data[q][keep].reshape(-1), rdata[q])


UCF = """2
2
0 0.0 0.0 0.0 2.0 0.01 1.0 Mn 0.0 0.0 1.0 1e-23 0 0 1
1 0.5 0.5 0.5 2.5 0.02 1.0 Au 0.0 0.0 -1.0 2e-23 0 0 1
"""

EXCH = """# exchange in the reference's unitcell format
exchange:
{
    MaxInteractions=3;
};
exchange_0_0:
{
    Num_Interactions=2;
    units="meV";
    UnitCell1 = [ 0.0 , 0.0 , 1.0 ];
    J1_1 = [ 1.0 , 0.0 , 0.0 ];
    J1_2 = [ 0.0 , 1.0 , 0.0 ];
    J1_3 = [ 0.0 , 0.0 , 1.0 ];
    UnitCell2 = [ 0.0 , 0.0 , -1.0 ];
    J2_1 = [ 1.0 , 0.0 , 0.0 ];
    J2_2 = [ 0.0 , 1.0 , 0.0 ];
    J2_3 = [ 0.0 , 0.0 , 1.0 ];
};
exchange_0_1:
{
    Num_Interactions=1;
    units="J";   // joules
    UnitCell1 = [ -0.6 , 0.4 , 0.0 ];
    J1_1 = [ -2e-21 , 1e-22 , 0.0 ];
    J1_2 = [ -1e-22 , -2e-21 , 0.0 ];
    J1_3 = [ 0.0 , 0.0 , -2e-21 ];
};
/* 1 -> 0 and 1 -> 1 */
exchange_1_0:
{
    Num_Interactions=1;
    units="joules";
    UnitCell1 = [ 0.6 , -0.4 , 0.0 ];
    J1_1 = [ -2e-21 , -1e-22 , 0.0 ];
    J1_2 = [ 1e-22 , -2e-21 , 0.0 ];
    J1_3 = [ 0.0 , 0.0 , -2e-21 ];
};
"""


def test_read_ucf_and_exch(tmp_path):
    (tmp_path / "a.ucf").write_text(UCF)
    (tmp_path / "a.exch").write_text(EXCH)
    nms, atoms = A.read_ucf(str(tmp_path / "a.ucf"))
    assert nms == 2 and len(atoms) == 2
    assert atoms[1]["mu"] == 2.5 and atoms[1]["element"] == "Au" and atoms[1]["init_spin"] == (0.0, 0.0, -1.0)
    assert atoms[0]["k1u"] == 1e-23 and atoms[0]["k1u_dir"] == (0.0, 0.0, 1.0)
    s1, s2, vec, J = A.read_exch(str(tmp_path / "a.exch"), nms)
    assert list(s1) == [0, 0, 0, 1] and list(s2) == [0, 0, 1, 0]
    # cell offsets rounded half away from zero (-0.6 -> -1, 0.4 -> 0)
    assert vec.tolist() == [[0, 0, 1], [0, 0, -1], [-1, 0, 0], [1, 0, 0]]
    assert J[0, 0, 0] == 1.0 * 1.602176565e-22 and J[2, 0, 1] == 1e-22
    s, _ = LT.from_reference_inputs(str(tmp_path / "a.ucf"), str(tmp_path / "a.exch"), (3, 3, 3))
    assert s.nspins == 54 and s.meta["nnz"] == 27 * 3 + 27 * 1


def test_read_ucf_with_mesh_points(tmp_path):
    (tmp_path / "m.ucf").write_text("1\n1\n0 0.0 0.0 0.0 0 0 0 1.5 0.1 1.0 Fe 1.0 0.0 0.0 0.0 0 0 1\n")
    nms, atoms = A.read_ucf(str(tmp_path / "m.ucf"), mesh_points=True)
    assert atoms[0]["mesh_point"] == (0, 0, 0) and atoms[0]["init_spin"] == (1.0, 0.0, 0.0)


@pytest.mark.parametrize("text,frag", [
    ("1\n1\n0 0 0 0 1e-6 0.1 1.0 Fe 0 0 1 0 0 0 1\n", "less than 1e-5"),
    ("1\n1\n0 0 0 0 1.5 0.1 1e6 Fe 0 0 1 0 0 0 1\n", "Gyromagnetic is greater"),
    ("1\n1\n0 0 0 0 1.5 0.1 1.0 Fe 0 0 1 0 0 0 2\n", "modulus of 1"),
    ("1\n1\n1 0 0 0 1.5 0.1 1.0 Fe 0 0 1 0 0 0 1\n", "species number"),
    ("1\n2\n0 0 0 0 1.5 0.1 1.0 Fe 0 0 1 0 0 0 1\n0 .5 .5 .5 2.0 0.1 1.0 Fe 0 0 1 0 0 0 1\n", "not consistent"),
    ("1\n2\n0 0 0 0 1.5 0.1 1.0 Fe 0 0 1 0 0 0 1\n", "ended early"),
    ("1\n0\n", "no atoms"),
])
def test_read_ucf_errors(tmp_path, text, frag):
    (tmp_path / "bad.ucf").write_text(text)
    with pytest.raises(A.AsdError) as e:
        A.read_ucf(str(tmp_path / "bad.ucf"))
    assert frag in str(e.value)


@pytest.mark.parametrize("text,frag", [
    ('exchange_0_0: { Num_Interactions=1; units="furlongs"; UnitCell1=[1,0,0]; J1_1=[1,0,0]; J1_2=[0,1,0]; '
     'J1_3=[0,0,1]; };', "not recognised"),
    ('exchange_0_0: { Num_Interactions=1; units="J"; J1_1=[1,0,0]; J1_2=[0,1,0]; J1_3=[0,0,1]; };', "vector"),
    ('exchange_0_0: { Num_Interactions=1; units="J"; UnitCell1=[1,0,0]; J1_1=[1,0,0]; J1_3=[0,0,1]; };', "J1_2"),
    ('exchange_0_0: { units="J"; };', "number of interactions"),
    ('exchange_0_0: { Num_Interactions=1; units="J ; };', "unterminated"),
    ('exchange_0_0 { Num_Interactions=0; };', "expected '='"),
])
def test_read_exch_errors(tmp_path, text, frag):
    (tmp_path / "bad.exch").write_text(text)
    with pytest.raises(A.AsdError) as e:
        A.read_exch(str(tmp_path / "bad.exch"), 1)
    assert frag in str(e.value)


def test_csr_exch_file_round_trip(tmp_path):
    s = LT.sc_ferromagnet((4, 3, 5), J2=3e-22)
    p = str(tmp_path / "csr_exch_mat.dat")
    A.write_csr_exch(p, s.xadj, s.adjncy, s.csr_val)
    xadj, adj, val = A.read_csr_exch(p, s.nspins)
    assert np.array_equal(xadj, s.xadj) and np.array_equal(adj, s.adjncy)
    assert np.array_equal(val[:, [0, 4, 8]], s.csr_val[:, [0, 4, 8]])
    with pytest.raises(A.AsdError):
        A.read_csr_exch(p, s.nspins + 1)             # first check of src/exch.cpp:77-81


REF_EXAMPLES = os.path.join(O.reference_dir(), "Examples")


@pytest.mark.skipif(not os.path.isdir(REF_EXAMPLES), reason="reference examples not present")
def test_reference_example_inputs_drive_the_builder():
    """The reference's own bcc-Fe example (two-atom cell, eight nearest neighbours across the
    two atoms) parses and builds a CSR with 8 entries per row; the CSR equals exchunitcell's."""
    d = os.path.join(REF_EXAMPLES, "MvsT", "bccFeNN")
    ucf = [f for f in os.listdir(d) if f.endswith(".ucf")][0]
    exch = [f for f in os.listdir(d) if f.endswith(".exch")][0]
    s, atoms = LT.from_reference_inputs(os.path.join(d, ucf), os.path.join(d, exch), (4, 4, 4))
    rows = np.diff(s.xadj)
    assert np.all(rows == 8)
    nms, _ = A.read_ucf(os.path.join(d, ucf))
    s1, s2, vec, J = A.read_exch(os.path.join(d, exch), nms)
    if HAVE_REF_BUILDERS:
        bonds = list(zip(s1, s2, vec, J))
        rx, ra, rv = O.ref_exchunitcell((4, 4, 4), (1, 1, 1), [a["mu"] for a in atoms], bonds, offdiag=True)
        assert np.array_equal(rx, s.xadj) and np.array_equal(ra, s.adjncy) and np.array_equal(rv, s.csr_val)


def test_spins_random_is_the_reference_marsaglia_on_its_mwc_stream():
    """asd_spins_random == the oracle's restatement of spins::setSpinsRandom bit for bit, and the
    oracle's MWC1616 == the reference's own Random::rand compiled from source."""
    for mwc in ((1, 101), (7, 107), (123456789, 987654321)):
        got, st = A.spins_random(2000, mwc)
        ref = O.spins_random(2000, mwc)
        assert np.array_equal(got, ref)
        assert np.allclose(np.linalg.norm(got, axis=1), 1.0, atol=1e-15)
        # the returned state continues the stream where the spins left it
        nxt, _ = A.spins_random(5, st)
        assert np.array_equal(nxt, O.spins_random(2005, mwc)[2000:])
    if os.path.exists(O.REF_SO):
        L = O.olib()
        L.orc_mwc_seed(7, 107)
        mine = np.array([L.orc_mwc_rand() for _ in range(5000)])
        assert np.array_equal(mine, O.ref_rand_stream(5000, (7, 107)))
    with pytest.raises(A.AsdError):
        A.spins_random(4, (0, 5))           # Random::seed rejects a zero seed


def test_spins_patterns():
    L = 3
    coords = np.array([(x, y, z) for x in range(L) for y in range(L) for z in range(L)], dtype=np.int32)
    for axis in range(3):
        s = A.spins_pattern(len(coords), axis, coords=coords)
        sign = np.where(coords.sum(axis=1) % 2 == 0, 1.0, -1.0)
        want = np.zeros((len(coords), 3))
        want[:, axis] = sign
        assert np.array_equal(s, want)
    init = np.array([[0.0, 0.0, 1.0], [0.6, 0.0, -0.8]])
    atom = np.arange(10, dtype=np.uint32) % 2
    s = A.spins_pattern(10, 3, atom_of_spin=atom, init_spin=init)
    assert np.array_equal(s, init[atom])
