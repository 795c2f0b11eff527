"""asd_magnetisation_noalloc: the magnetisation for callers that cannot allocate device memory
(under a pool allocator that owns the device, or in a loop that must avoid cudaFree's
device-wide synchronisation).  Its scratch is a static device array, so the checks here are
that two calls in a row through the C ABI agree with the handle-based asd_magnetisation (which
allocates its scratch at asd_create) and with the mean of each sublattice's spins computed on
the host, also at sizes where every block strides over several spins, with 16 sublattices, with
ids beyond nsub (left out) and with no sublattice array.  Collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

import asd_b200 as A
import asd_lattice as LT

pytestmark = pytest.mark.gpu

TOL = 1e-14   # the magnetisation tolerance used by the other GPU tests


def test_noalloc_magnetisation_matches_handle_magnetisation(gpu):
    import torch

    lib = A.load_library()
    s = LT.bct2_antiferromagnet(6, T=300.0)            # 2 sublattices, 432 spins
    with A.Handle(A.RunParams(precision=A.FP64_PLAIN, seed=3), s) as h:
        h.set_spins(LT.random_spins(s.nspins, 5))
        h.step(20)
        spins = h.get_spins()
        want = h.magnetisation()[0]                     # existing entry point, [nsub, 3]
    nsub = want.shape[0]
    sub = np.arange(s.nspins, dtype=np.uint32) % 2    # atom t -> sublattice t
    d_spins = torch.tensor(spins.reshape(-1), dtype=torch.float64, device="cuda")
    d_sub = torch.tensor(sub.astype(np.int32), dtype=torch.int32, device="cuda")
    for call in range(2):
        d_out = torch.full((nsub * 3,), float("nan"), dtype=torch.float64, device="cuda")
        rc = lib.asd_magnetisation_noalloc(C.c_void_p(d_spins.data_ptr()), s.nspins, C.c_void_p(d_sub.data_ptr()),
                                           nsub, C.c_void_p(d_out.data_ptr()), None)
        assert rc == A.ASD_OK
        torch.cuda.synchronize()
        got = d_out.cpu().numpy().reshape(nsub, 3)
        assert np.abs(got - want).max() <= TOL, (call, got, want)
        host = np.stack([spins[sub == q].mean(0) for q in range(nsub)])
        assert np.abs(got - host).max() <= 1e-13, (call, got, host)


def noalloc(spins, sub, nsub):
    import torch
    lib = A.load_library()
    d_spins = torch.tensor(spins.reshape(-1), dtype=torch.float64, device="cuda")
    d_sub = None if sub is None else torch.tensor(sub.astype(np.int32), dtype=torch.int32, device="cuda")
    outs = []
    for call in range(2):
        d_out = torch.full((nsub * 3,), float("nan"), dtype=torch.float64, device="cuda")
        rc = lib.asd_magnetisation_noalloc(C.c_void_p(d_spins.data_ptr()), spins.shape[0],
                                           None if d_sub is None else C.c_void_p(d_sub.data_ptr()), nsub,
                                           C.c_void_p(d_out.data_ptr()), None)
        assert rc == A.ASD_OK
        torch.cuda.synchronize()
        outs.append(d_out.cpu().numpy().reshape(nsub, 3))
    return outs


@pytest.mark.parametrize("n,nsub", [(600_001, 16), (524_289, 5), (1_000, 1)])
def test_noalloc_large_ragged_against_host_means(gpu, n, nsub):
    """n above 2048 x 256 spins: each block strides over several spins; ids up to nsub + 2, the
    ones >= nsub left out of every sum."""
    rng = np.random.default_rng(n)
    spins = LT.random_spins(n, 7)
    sub = rng.integers(0, nsub + 2, n).astype(np.uint32)
    host = np.stack([spins[sub == q].mean(0) for q in range(nsub)])
    for got in noalloc(spins, sub, nsub):
        assert np.abs(got - host).max() <= 1e-12, np.abs(got - host).max()


def test_noalloc_without_sublattices(gpu):
    spins = LT.random_spins(777_777, 9)
    for got in noalloc(spins, None, 1):
        assert np.abs(got[0] - spins.mean(0)).max() <= 1e-12


def test_noalloc_rejects_sizes_beyond_its_scratch(gpu):
    lib = A.load_library()
    assert lib.asd_magnetisation_noalloc(C.c_void_p(16), 10, None, 17, C.c_void_p(16), None) == A.ASD_EINVAL
    assert lib.asd_magnetisation_noalloc(None, 10, None, 1, C.c_void_p(16), None) == A.ASD_EINVAL
