"""Shared helpers of the GPU parity tests (CUDA path through the C ABI vs the oracle)."""
import numpy as np
import torch

from oracle import afqmc as O


def rel_err(a, b, atol=1e-13):
    """||a-b||_inf / max(||a||_inf, ||b||_inf, atol/rtol-floor): the reference's Approx metric
    (tests/test_common.hpp:384-438) with an absolute floor, so roundoff-level values (1e-17) that
    one side computes as exact zeros do not count as relative errors of 1."""
    a = np.asarray(a).ravel()
    b = np.asarray(b).ravel()
    d = np.max(np.abs(a - b)) if a.size else 0.0
    v = max(np.max(np.abs(a)) if a.size else 0.0, np.max(np.abs(b)) if b.size else 0.0)
    if d <= atol:
        return 0.0
    return d / v if v > 0 else d


def to_dev(a, dtype=torch.complex128):
    return torch.from_numpy(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


def to_host(t):
    torch.cuda.synchronize()
    return t.detach().cpu().numpy()


def rand_c(rs, *shape, scale=1.0):
    return scale * (rs.standard_normal(shape) + 1j * rs.standard_normal(shape))


def make_pair(wl):
    """(device HamiltonianOperations, oracle Real3IndexFactorization, oracle NOMSD)."""
    from safire_b200 import afqmc as A
    dham = A.HamiltonianOperations(wl.walker_type, wl.M, wl.nup, wl.ndn, wl.Likn, wl.hij, wl.E0,
                                   wl.PsiT)
    oham = O.Real3IndexFactorization(wl.walker_type, wl.M, wl.nup, wl.ndn, wl.Likn, wl.hij, wl.E0,
                                     wl.PsiT)
    return dham, oham, O.NOMSD(oham, wl.PsiT)
