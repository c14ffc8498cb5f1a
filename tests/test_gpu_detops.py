"""det_ops through the C ABI on the GPU vs the reference golden vectors and the oracle."""
import numpy as np
import pytest
import torch

from oracle import afqmc as O
from tests.golden import sdet_ops_golden as g
from tests.gpu_helpers import rand_c, rel_err, to_dev, to_host

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _A():
    from safire_b200 import afqmc as A
    return A


def test_golden_log_overlap(cuda):
    A = _A()
    B = to_dev(np.repeat(g.M_B[None], g.NWALK, 0))
    ov = torch.zeros(g.NWALK, dtype=torch.complex128, device=cuda)
    A.det_ops.Log_Overlap(to_dev(g.M_A), B, ov)
    assert g.approx(to_host(ov), np.full(g.NWALK, g.OV_BASE))
    B2 = to_dev(np.repeat(g.M_B[None, :3, :2], g.NWALK, 0))
    ov2 = torch.zeros(g.NWALK, dtype=torch.complex128, device=cuda)
    A.det_ops.Log_Overlap(to_dev(g.M_A[:2, :3]), B2, ov2)
    assert g.approx(to_host(ov2), np.full(g.NWALK, g.OV2_BASE))


@pytest.mark.parametrize("compact", [True, False])
def test_golden_mixed_density_matrix(cuda, compact):
    A = _A()
    for a, b, ref in [(g.M_A, g.M_B, g.VC_REF if compact else g.V_REF),
                      (g.M_A[:2, :3], g.M_B[:3, :2], g.VC_REF_2 if compact else g.V_REF_2)]:
        N, M = a.shape
        B = to_dev(np.repeat(b[None], g.NWALK, 0))
        G = torch.zeros((g.NWALK,) + ((N, M) if compact else (M, M)), dtype=torch.complex128,
                        device=cuda)
        ov = torch.zeros(g.NWALK, dtype=torch.complex128, device=cuda)
        A.det_ops.MixedDensityMatrix(to_dev(a), B, G, ov, compact=compact)
        assert g.approx(to_host(G), np.repeat(ref[None], g.NWALK, 0))
    assert g.approx(to_host(ov), np.full(g.NWALK, g.OV2_BASE))


def test_golden_inverse_logdet(cuda):
    A = _A()
    Am = to_dev(np.repeat(g.INV_A[None], g.NWALK, 0))
    inv = torch.zeros_like(Am)
    ld = torch.zeros(g.NWALK, dtype=torch.complex128, device=cuda)
    A.det_ops.inverse_logdet(Am, inv, ld)
    assert g.approx(to_host(inv), np.repeat(g.INV_REF[None], g.NWALK, 0))
    assert g.approx(to_host(ld), np.full(g.NWALK, g.LOGDET_INV_REF))


def test_golden_orthogonalize(cuda):
    A = _A()
    Q = to_dev(np.repeat(g.M_B[None], g.NWALK, 0))
    ld = torch.zeros(g.NWALK, dtype=torch.complex128, device=cuda)
    A.det_ops.orthogonalize(Q, ld)
    q = to_host(Q)
    # test_sdet_ops.cpp:296-304: Log_Overlap(Q, Q) == 0
    ov = torch.zeros(g.NWALK, dtype=torch.complex128, device=cuda)
    A.det_ops.Log_Overlap(to_dev(np.ascontiguousarray(q[0].conj().T)), Q, ov)
    assert g.approx(to_host(ov), np.zeros(g.NWALK))
    qo = np.repeat(g.M_B[None], g.NWALK, 0).copy()
    ldo = np.zeros(g.NWALK, complex)
    O.orthogonalize(qo, ldo)
    assert rel_err(q, qo) < TOL
    assert rel_err(to_host(ld), ldo) < TOL


def test_singular_inverse_is_zero(cuda):
    A = _A()
    m = np.array([[1, 2], [2, 4]], dtype=complex)
    Am = to_dev(m[None])
    inv = torch.ones_like(Am)
    ld = torch.zeros(1, dtype=torch.complex128, device=cuda)
    A.det_ops.inverse_logdet(Am, inv, ld)
    assert np.all(to_host(inv) == 0)
    ldo = np.zeros(1, complex)
    O.inverse_logdet(m[None], ldo)
    assert abs(to_host(ld)[0].real - ldo[0].real) < 1e-9


@pytest.mark.parametrize("N", [1, 2, 7, 8, 9, 16, 17, 32, 33, 50, 52, 53, 64, 65, 70])
def test_random_inverse_logdet_sizes(cuda, N):
    """Every size class of the register-resident kernel (N <= 64) and the shared-memory kernel
    (N > 64): inverse and accumulated log det against the oracle's getrf/getri."""
    A = _A()
    rs = np.random.default_rng(100 + N)
    W = 5
    m = rand_c(rs, W, N, N)
    ld0 = rand_c(rs, W) * 0.5
    Am = to_dev(m)
    inv = torch.zeros_like(Am)
    ld = to_dev(ld0.copy())
    A.det_ops.inverse_logdet(Am, inv, ld)
    ldo = ld0.copy()
    invo = O.inverse_logdet(m, ldo)
    assert rel_err(to_host(inv), invo) < TOL
    assert rel_err(to_host(ld), ldo) < TOL


@pytest.mark.parametrize("N", [3, 16, 31, 33, 52, 53, 64, 66])
def test_random_log_overlap_sizes(cuda, N):
    """LU-only log det (Log_Overlap) in every size class, against the oracle."""
    A = _A()
    rs = np.random.default_rng(300 + N)
    W, M = 6, N + 5
    psi = rand_c(rs, N, M) / np.sqrt(M)
    S = rand_c(rs, W, M, N) / np.sqrt(M)
    ov = to_dev(rand_c(rs, W, scale=0.1))
    ovo = to_host(ov).copy()
    A.det_ops.Log_Overlap(to_dev(psi), to_dev(S), ov)
    O.Log_Overlap(psi, S, ovo)
    assert rel_err(to_host(ov), ovo) < TOL


@pytest.mark.parametrize("W,M,N", [(7, 32, 8), (33, 40, 13), (4, 200, 50)])
def test_random_density_matrix_and_overlap(cuda, W, M, N):
    A = _A()
    rs = np.random.default_rng(W * 1000 + M + N)
    psi = rand_c(rs, N, M) / np.sqrt(M)
    S = rand_c(rs, W, M, N) / np.sqrt(M)
    for compact in (True, False):
        G = torch.zeros((W, N, M) if compact else (W, M, M), dtype=torch.complex128, device=cuda)
        ov = to_dev(rand_c(rs, W, scale=0.1))
        ovo = to_host(ov).copy()
        A.det_ops.MixedDensityMatrix(to_dev(psi), to_dev(S), G, ov, compact=compact)
        Go = O.MixedDensityMatrix(psi, S.copy(), ovo, compact=compact)
        assert rel_err(to_host(G), Go) < TOL
        assert rel_err(to_host(ov), ovo) < TOL
    ov = torch.zeros(W, dtype=torch.complex128, device=cuda)
    A.det_ops.Log_Overlap(to_dev(psi), to_dev(S), ov)
    ovo = np.zeros(W, complex)
    O.Log_Overlap(psi, S, ovo)
    assert rel_err(to_host(ov), ovo) < TOL


def test_strided_walker_rows(cuda):
    """S passed with a walker stride > M*N, like rows of the walker buffer."""
    A = _A()
    rs = np.random.default_rng(5)
    W, M, N, extra = 6, 24, 5, 11
    psi = rand_c(rs, N, M)
    rows = rand_c(rs, W, M * N + extra)
    buf = to_dev(rows)
    S = buf[:, :M * N].unflatten(1, (M, N))
    ov = torch.zeros(W, dtype=torch.complex128, device=cuda)
    A.det_ops.Log_Overlap(to_dev(psi), S, ov)
    ovo = np.zeros(W, complex)
    O.Log_Overlap(psi, rows[:, :M * N].reshape(W, M, N), ovo)
    assert rel_err(to_host(ov), ovo) < TOL


@pytest.mark.parametrize("W,M,N", [(5, 32, 8), (3, 200, 50)])
def test_random_orthogonalize(cuda, W, M, N):
    A = _A()
    rs = np.random.default_rng(M + N)
    S = rand_c(rs, W, M, N)
    Sd = to_dev(S)
    ld = torch.zeros(W, dtype=torch.complex128, device=cuda)
    A.det_ops.orthogonalize(Sd, ld)
    So = S.copy()
    ldo = np.zeros(W, complex)
    O.orthogonalize(So, ldo)
    assert rel_err(to_host(Sd), So) < TOL
    assert rel_err(to_host(ld), ldo) < TOL


@pytest.mark.parametrize("W,M,N,order", [(4, 32, 8, 6), (3, 64, 10, 4), (2, 200, 50, 6)])
def test_random_propagate(cuda, W, M, N, order):
    A = _A()
    rs = np.random.default_rng(order + M)
    S = rand_c(rs, W, M, N)
    P1 = np.eye(M) + rand_c(rs, M, M, scale=0.01)
    V = rand_c(rs, W, M, M, scale=0.05)
    Sd = to_dev(S)
    A.det_ops.Propagate(Sd, to_dev(P1), to_dev(V), order)
    So = S.copy()
    O.propagate_impl(So, P1, V, order)
    assert rel_err(to_host(Sd), So) < TOL
