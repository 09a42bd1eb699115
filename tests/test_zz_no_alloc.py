"""The allocation-free survivor count, pspin_fmc_survivors_static.

Callers that cannot allocate device memory (hosts whose own pool owns all
device memory, plugins handed only device pointers) get the FMC survivor
count through this entry point, whose scratch is a static device array.  Its result must equal the existing entry point's
(pspin_fmc_mask: the popcount of the mask it builds, and the per-channel
counts read off that mask), on two calls in a row since the calls share the
array.  Collected last so that a failure here leaves every other test run.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _static_counts(ps, torch, N, w, gamma):
    lib = ps.load_library()
    d_w = torch.tensor(w, dtype=torch.float64, device="cuda")
    d_out = torch.full((4,), -1, dtype=torch.int64, device="cuda")
    rc = lib.pspin_fmc_survivors_static(N, ctypes.c_void_p(d_w.data_ptr()), float(gamma),
                                        ctypes.c_void_p(d_out.data_ptr()), None)
    assert rc == 0, lib.pspin_last_error()
    torch.cuda.synchronize()
    return d_out.cpu().numpy()


@pytest.mark.parametrize("N,fmc,seed,gamma", [(10, 1, 0, 1.0), (32, 2, 42, 0.1), (64, 2, 42, 0.1),
                                              (24, 2, 9, 1.0 / 46), (48, 1, 0, 2.0), (128, 2, 7, 0.05),
                                              (256, 1, 0, 1.0)])
def test_static_count_matches_existing_entry_point(ps, orc, N, fmc, seed, gamma):
    torch = pytest.importorskip("torch")
    w = orc.omega(N, fmc, seed)
    mask, n_active = ps.fmc_mask(N, w, gamma)
    per_ch = [int(np.count_nonzero(mask == (1 << c))) for c in range(3)]
    for _ in range(2):   # the scratch array keeps the previous call's rows
        got = _static_counts(ps, torch, N, w, gamma)
        assert got[0] == n_active
        assert list(got[1:]) == per_ch


def test_static_count_rejects_too_large_n(ps):
    torch = pytest.importorskip("torch")
    lib = ps.load_library()
    d_w = torch.zeros(2048, dtype=torch.float64, device="cuda")
    d_out = torch.zeros(4, dtype=torch.int64, device="cuda")
    rc = lib.pspin_fmc_survivors_static(2048, ctypes.c_void_p(d_w.data_ptr()), 0.1,
                                        ctypes.c_void_p(d_out.data_ptr()), None)
    assert rc == 1
    assert b"static scratch" in lib.pspin_last_error()
