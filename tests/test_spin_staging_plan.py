"""Host-side check of the neighbour-spin staging plan (asd_plan_spin_spans) against the buffers
the fused stage kernel touches: every local slot maps back to its global column, every span
is 16-byte aligned and inside the padded spin allocation, slots fit the shared-memory budget.
Runs without a GPU."""
import ctypes as C

import numpy as np
import pytest

import asd_b200 as A
import asd_lattice as LT

SPIN_PAD = 8
SMEM_LIMIT = 227 * 1024


def sell_words(xadj, adj, colbits, rng):
    """SELL-32 slices and typed words laid out as the library lays them out: entry
    (slice s, k, lane) at slice_ptr[s] + 32k + lane; padding points at the row itself (or 0
    past the last row) with tensor id 0."""
    n = len(xadj) - 1
    ns = (n + 31) // 32
    rowlen = np.diff(xadj)
    sp = np.zeros(ns + 1, dtype=np.uint32)
    for s in range(ns):
        sp[s + 1] = sp[s] + 32 * rowlen[32 * s: 32 * s + 32].max()
    w = np.zeros(sp[-1], dtype=np.uint32)
    ntypes = 1 << (32 - colbits)
    for s in range(ns):
        wd = (sp[s + 1] - sp[s]) // 32
        for lane in range(32):
            r = 32 * s + lane
            for k in range(wd):
                e = sp[s] + 32 * k + lane
                if r < n and k < rowlen[r]:
                    col, t = adj[xadj[r] + k], rng.integers(1, ntypes)
                else:
                    col, t = (r if r < n else 0), 0
                w[e] = col | (t << colbits)
    return sp, w


def plan(n, sp, w, colbits, elem, block):
    lib = A.load_library()
    ns = len(sp) - 1
    nblk = (ns + block // 32 - 1) // (block // 32)
    ptr = np.zeros(nblk + 1, dtype=np.uint32)
    nsp, slots = C.c_uint32(), C.c_uint32()
    u = lambda a: a.ctypes.data_as(C.POINTER(C.c_uint32))
    rc = lib.asd_plan_spin_spans(n, ns, u(sp), u(w), colbits, elem, block, u(ptr), None, 0, None, C.byref(nsp),
                                 C.byref(slots))
    assert rc == 0
    spans = np.zeros((max(nsp.value, 1), 4), dtype=np.uint32)
    lw = np.zeros_like(w)
    rc = lib.asd_plan_spin_spans(n, ns, u(sp), u(w), colbits, elem, block, u(ptr), u(spans), nsp.value, u(lw),
                                 C.byref(nsp), C.byref(slots))
    assert rc == 0
    return ptr, spans[: nsp.value], lw, slots.value


def _systems():
    return [LT.bct2_antiferromagnet(6), LT.sc_ferromagnet((9, 7, 5)), LT.film_dia(24, 20, 3, dipole=False),
            LT.sc_ferromagnet((3, 3, 3), pbc=(0, 0, 0))]


@pytest.fixture(scope="module")
def lib():
    return A.load_library()


@pytest.mark.parametrize("k", range(4))
@pytest.mark.parametrize("block", [64, 128, 256])
@pytest.mark.parametrize("elem", [4, 8])
def test_plan_maps_every_slot_back_to_its_column(lib, k, block, elem):
    s = _systems()[k]
    if s.exch == A.EXCH_DIA:   # the film builder returns DIA; rebuild its CSR
        xadj, adj, _ = LT.build_csr(s.meta["dim"], (1, 1, 0), [s.materials[0].mu], [0] * 18, [0] * 18,
                                    list(LT.SC_NN) + list(LT.SC_NNN), [LT._iso(1e-21)] * 18)
    else:
        xadj, adj = s.xadj, s.adjncy
    n = len(xadj) - 1
    colbits = 28
    sp, w = sell_words(xadj, adj, colbits, np.random.default_rng(k))
    ptr, spans, lw, slots = plan(n, sp, w, colbits, elem, block)
    align = 16 // elem
    mask = (1 << colbits) - 1
    spb = block // 32
    nblk = len(ptr) - 1
    staged = 0
    for b in range(nblk):
        e0, e1 = sp[b * spb], sp[min((b + 1) * spb, len(sp) - 1)]
        bs = spans[ptr[b]: ptr[b + 1]]
        if len(bs) == 0:
            assert np.array_equal(lw[e0:e1], w[e0:e1])
            continue
        staged += 1
        assert len(bs) <= 24
        off = 0
        for st, ln, o, z in bs:
            assert st % align == 0 and ln % align == 0 and ln > 0 and z == 0
            assert st + ln <= n + SPIN_PAD                      # inside the padded allocation
            assert o == off and o % align == 0                  # 16-byte aligned shared-memory slots
            off += ln
        assert off <= slots and 3 * slots * elem <= 64 * 1024
        assert np.all(bs[1:, 0] >= bs[:-1, 0] + bs[:-1, 1])    # disjoint, ascending
        loc = lw[e0:e1] & mask
        glob = w[e0:e1] & mask
        assert np.array_equal(lw[e0:e1] >> colbits, w[e0:e1] >> colbits)   # tensor ids kept
        idx = np.searchsorted(bs[:, 2], loc, side="right") - 1
        assert np.all(loc < bs[idx, 2] + bs[idx, 1])
        assert np.array_equal(bs[idx, 0] + (loc - bs[idx, 2]), glob)
    assert staged == nblk            # these lattices are local enough for every block
    # the kernel's shared memory: table (<= 12 KB) + words + spins
    words_max = max(int(sp[min((b + 1) * spb, len(sp) - 1)] - sp[b * spb]) for b in range(nblk))
    assert 12 * 1024 + 4 * words_max + 3 * slots * elem <= SMEM_LIMIT


def test_plan_falls_back_for_scattered_columns(lib):
    """A random graph has no locality: blocks exceed the span budget and keep global columns."""
    rng = np.random.default_rng(1)
    n, z = 20000, 12
    adj = rng.integers(0, n, size=n * z).astype(np.uint32)
    xadj = (np.arange(n + 1) * z).astype(np.uint32)
    sp, w = sell_words(xadj, adj, 28, rng)
    ptr, spans, lw, slots = plan(n, sp, w, 28, 4, 256)
    assert len(spans) == 0 and np.array_equal(lw, w)


def test_plan_rejects_bad_arguments(lib):
    u = lambda a: a.ctypes.data_as(C.POINTER(C.c_uint32))
    sp = np.array([0, 32], dtype=np.uint32)
    w = np.full(32, 40, dtype=np.uint32)        # column 40 >= n
    ptr = np.zeros(2, dtype=np.uint32)
    a, b = C.c_uint32(), C.c_uint32()
    assert lib.asd_plan_spin_spans(32, 1, u(sp), u(w), 28, 4, 64, u(ptr), None, 0, None, C.byref(a), C.byref(b)) \
        == A.ASD_EINVAL
    assert lib.asd_plan_spin_spans(32, 1, u(sp), u(w), 28, 6, 64, u(ptr), None, 0, None, C.byref(a), C.byref(b)) \
        == A.ASD_EINVAL
