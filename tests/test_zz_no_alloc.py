"""asd_magnetisation_noalloc: the magnetisation for callers that cannot allocate device memory
(inside a CUDA-graph capture, under a pool allocator that owns the device, or in a loop that
must avoid cudaFree's device-wide synchronisation).  Its scratch is a static device array,
so the check here is that two calls in a row through the C ABI agree with the handle-based
asd_magnetisation, which allocates its scratch at asd_create.  Collected last on purpose."""
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


def test_noalloc_rejects_sizes_beyond_its_scratch(gpu):
    lib = A.load_library()
    assert lib.asd_magnetisation_noalloc(C.c_void_p(16), 10, None, 17, C.c_void_p(16), None) == A.ASD_EINVAL
    assert lib.asd_magnetisation_noalloc(None, 10, None, 1, C.c_void_p(16), None) == A.ASD_EINVAL
