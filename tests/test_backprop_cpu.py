"""Back-propagation host logic on the CPU: the comb's slot map, the oracle's backward
propagation as the adjoint of the forward one, and the path-restoration factors."""
import numpy as np

from oracle import afqmc as O
from oracle import backprop as OB
from safire_b200.backprop import slot_map


def test_slot_map_matches_the_comb_restatement():
    rs = np.random.default_rng(0)
    for _ in range(50):
        W = int(rs.integers(1, 40))
        w = rs.random(W) * (rs.random(W) > 0.3)
        if w.sum() == 0:
            w[0] = 1.0
        rng = O.HostRandomGenerator(int(rs.integers(1, 1 << 30)))
        off = O.comb(rng, w, W)
        assert np.array_equal(slot_map(off), O.single_rank_slot_map(off))


def _case(seed, W=3, M=6, N=2):
    rs = np.random.default_rng(seed)
    P1 = np.linalg.qr(rs.standard_normal((M, M)) + 1j * rs.standard_normal((M, M)))[0]
    P1 = P1 * 0.9 + 0.1 * np.eye(M)
    V = 0.1 * (rs.standard_normal((W, M, M)) + 1j * rs.standard_normal((W, M, M)))
    A = rs.standard_normal((W, M, N)) + 1j * rs.standard_normal((W, M, N))
    S = rs.standard_normal((W, M, N)) + 1j * rs.standard_normal((W, M, N))
    return P1, V, A, S


def test_backward_step_is_the_adjoint_of_the_forward_step():
    """A^H (P1 e^{iV} P1 S) = (P1^H e^{-iV^H} P1^H A)^H S for the order-6 series, and the
    orthogonalisation that ends the backward pass leaves the density matrix unchanged."""
    P1, V, A, S = _case(1)
    fwd = S.copy()
    O.propagate_impl(fwd, P1, V, 6, "N")
    refs = [A.copy()]
    OB.back_propagate(refs, [P1], [V[None]], 6, nstab=10)  # ni = 0: one QR at the end
    bwd = A.copy()
    T = np.matmul(P1.conj().T, bwd)
    O.apply_expM(V, T, 6, "H")
    bwd = np.matmul(P1.conj().T, T)
    lhs = np.matmul(np.conj(np.swapaxes(A, 1, 2)), fwd)
    rhs = np.matmul(np.conj(np.swapaxes(bwd, 1, 2)), S)
    assert np.allclose(lhs, rhs, atol=1e-12)
    w = np.array([0.5, 1.0, 2.0 + 0.1j])
    G_orth = OB.bp_onerdm(refs, [S], w)
    G_raw = OB.bp_onerdm([bwd], [S], w)
    assert np.allclose(G_orth, G_raw, atol=1e-12)


def test_weight_factors():
    props0 = np.zeros((4, 11), complex)
    props1 = np.zeros((4, 11), complex)
    props0[:, 1] = [1.0, np.exp(0.3j), 0.0, 1.0]
    ph = np.exp(-0.2j)
    props1[:, 1] = props0[:, 1] * ph
    props1[3, 1] = 0.0  # killed in this step
    props1[:, 10] = [0.4, 2.0, 0.1, 0.1]  # dtheta; cos(2.0) < 0
    f = OB.weight_factors(props0, props1, 1, 10)
    assert np.isclose(f[0], ph / np.cos(0.4))
    assert f[1] == 0 and f[2] == 0 and f[3] == 0
