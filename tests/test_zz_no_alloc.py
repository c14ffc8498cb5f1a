"""afqmc_log_overlap_noalloc: the log-overlap entry point for callers that cannot allocate device
memory (its scratch is a fixed array inside the library).  It must give the same result as
afqmc_log_overlap, call after call, accumulate into ovlp as that entry point does, allocate no
device memory, and reject sizes beyond its fixed scratch.  Collected last so that a run stopping
at the first failure has run every other test before it."""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

CU_MEMPOOL_ATTR_RESERVED_MEM_CURRENT = 5
CU_MEMPOOL_ATTR_USED_MEM_CURRENT = 7
CU_MEMPOOL_ATTR_USED_MEM_HIGH = 8


def _call(name, psi, S, ov):
    from safire_b200 import capi
    W, M, N = S.shape
    return capi.lib().__getattr__(name)(C.c_void_p(psi.data_ptr()), C.c_void_p(S.data_ptr()),
                                        S.stride(0), C.c_void_p(ov.data_ptr()), W, M, N,
                                        C.c_void_p(torch.cuda.current_stream().cuda_stream))


def _inputs(cuda, W, M, N, seed):
    rs = np.random.default_rng(seed)
    psi = torch.from_numpy((rs.standard_normal((N, M)) + 1j * rs.standard_normal((N, M)))
                           / np.sqrt(M)).to(cuda)
    S = torch.from_numpy((rs.standard_normal((W, M, N)) + 1j * rs.standard_normal((W, M, N)))
                         / np.sqrt(M)).to(cuda)
    # ovlp is accumulated into (+=), as in the reference: start both entry points from the same
    # non-zero values
    ov0 = torch.from_numpy(rs.standard_normal(W) + 1j * rs.standard_normal(W)).to(cuda)
    return psi, S, ov0


class _DriverPool:
    """The device's default memory pool through the driver API (the pool the stream-ordered
    allocator of the allocating entry point draws from)."""

    def __init__(self, device_index):
        self.cu = C.CDLL("libcuda.so.1")
        dev = C.c_int()
        assert self.cu.cuDeviceGet(C.byref(dev), device_index) == 0
        self.pool = C.c_void_p()
        assert self.cu.cuDeviceGetDefaultMemPool(C.byref(self.pool), dev) == 0

    def get(self, attr):
        v = C.c_uint64()
        assert self.cu.cuMemPoolGetAttribute(self.pool, attr, C.byref(v)) == 0
        return v.value

    def reset_high(self):
        z = C.c_uint64(0)
        assert self.cu.cuMemPoolSetAttribute(self.pool, CU_MEMPOOL_ATTR_USED_MEM_HIGH,
                                             C.byref(z)) == 0


@pytest.mark.parametrize("W,M,N", [(40, 48, 10), (2, 96, 80)],
                         ids=["N10_register_path", "N80_shared_memory_path"])
def test_noalloc_matches_allocating_entry_point(cuda, W, M, N):
    """N = 10 runs the register-resident Gauss-Jordan kernel, N = 80 the shared-memory one."""
    psi, S, ov0 = _inputs(cuda, W, M, N, 21 + N)
    ref = ov0.clone()
    assert _call("afqmc_log_overlap", psi, S, ref) == 0
    for _ in range(2):  # two calls in a row share the fixed scratch
        out = ov0.clone()
        assert _call("afqmc_log_overlap_noalloc", psi, S, out) == 0
        torch.cuda.synchronize()
        d = (out - ref).abs().max().item()
        assert d <= 1e-10 * max(1.0, ref.abs().max().item()), d
        # the accumulation: out - ov0 is the log-overlap itself, non-zero
        assert (out - ov0).abs().min().item() > 0


def test_noalloc_allocates_nothing(cuda):
    """Around three calls (after a first one has loaded the kernels; every tensor allocated
    beforehand): the default memory pool's usage high-water mark stays where a reset put it (its
    current usage), its reservation is unchanged, and the device's free memory is unchanged."""
    W, M, N = 64, 64, 16
    psi, S, ov0 = _inputs(cuda, W, M, N, 5)
    outs = [ov0.clone() for _ in range(4)]
    assert _call("afqmc_log_overlap_noalloc", psi, S, outs[3]) == 0
    torch.cuda.synchronize()
    pool = _DriverPool(torch.cuda.current_device())
    pool.reset_high()
    used0 = pool.get(CU_MEMPOOL_ATTR_USED_MEM_CURRENT)
    reserved0 = pool.get(CU_MEMPOOL_ATTR_RESERVED_MEM_CURRENT)
    free0, _ = torch.cuda.mem_get_info()
    for k in range(3):
        assert _call("afqmc_log_overlap_noalloc", psi, S, outs[k]) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert pool.get(CU_MEMPOOL_ATTR_USED_MEM_HIGH) == used0
    assert pool.get(CU_MEMPOOL_ATTR_RESERVED_MEM_CURRENT) == reserved0
    assert free1 == free0
    for k in range(3):
        assert torch.equal(outs[k], outs[3])


def test_noalloc_rejects_oversized_calls(cuda):
    from safire_b200 import capi
    W, M, N = 300, 60, 50  # W*N*N = 750000 > 524288
    psi = torch.zeros((N, M), dtype=torch.complex128, device=cuda)
    S = torch.zeros((W, M, N), dtype=torch.complex128, device=cuda)
    out = torch.zeros(W, dtype=torch.complex128, device=cuda)
    st = _call("afqmc_log_overlap_noalloc", psi, S, out)
    assert st == 2  # AFQMC_ERR_SHAPE
    assert b"524288" in capi.lib().afqmc_last_error()
