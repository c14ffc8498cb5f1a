"""afqmc_log_overlap_noalloc: the log-overlap entry point for callers that cannot allocate device
memory (its scratch is a fixed array inside the library).  It must give the same result as
afqmc_log_overlap, call after call, and reject sizes beyond its fixed scratch.  Collected last so
that a run stopping at the first failure has run every other test before it."""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _call(name, psi, S, ov):
    from safire_b200 import capi
    W, M, N = S.shape
    return capi.lib().__getattr__(name)(C.c_void_p(psi.data_ptr()), C.c_void_p(S.data_ptr()),
                                        S.stride(0), C.c_void_p(ov.data_ptr()), W, M, N,
                                        C.c_void_p(torch.cuda.current_stream().cuda_stream))


def test_noalloc_matches_allocating_entry_point(cuda):
    rs = np.random.default_rng(21)
    W, M, N = 40, 48, 10
    psi = torch.from_numpy((rs.standard_normal((N, M)) + 1j * rs.standard_normal((N, M)))
                           / np.sqrt(M)).to(cuda)
    S = torch.from_numpy((rs.standard_normal((W, M, N)) + 1j * rs.standard_normal((W, M, N)))
                         / np.sqrt(M)).to(cuda)
    ref = torch.zeros(W, dtype=torch.complex128, device=cuda)
    assert _call("afqmc_log_overlap", psi, S, ref) == 0
    for _ in range(2):  # two calls in a row share the fixed scratch
        out = torch.zeros(W, dtype=torch.complex128, device=cuda)
        assert _call("afqmc_log_overlap_noalloc", psi, S, out) == 0
        torch.cuda.synchronize()
        d = (out - ref).abs().max().item()
        assert d <= 1e-10 * max(1.0, ref.abs().max().item()), d


def test_noalloc_rejects_oversized_calls(cuda):
    from safire_b200 import capi
    W, M, N = 300, 60, 50  # W*N*N = 750000 > 524288
    psi = torch.zeros((N, M), dtype=torch.complex128, device=cuda)
    S = torch.zeros((W, M, N), dtype=torch.complex128, device=cuda)
    out = torch.zeros(W, dtype=torch.complex128, device=cuda)
    st = _call("afqmc_log_overlap_noalloc", psi, S, out)
    assert st == 2  # AFQMC_ERR_SHAPE
    assert b"524288" in capi.lib().afqmc_last_error()
