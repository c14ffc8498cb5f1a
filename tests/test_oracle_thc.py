"""The THC restatement (oracle/thc.py, THCOps) against the Cholesky one (oracle/afqmc.py,
Real3IndexFactorization) on the Cholesky vectors the THC factors stand for: with Z = Luv Luv^T
the two factorisations are the same Hamiltonian, so vbias, vHS, the energy and the one-body
propagator agree to rounding."""
import numpy as np
import pytest

from oracle import afqmc as O
from oracle import thc as T
from safire_b200.synth import CLOSED, COLLINEAR, make_thc_system


def _G(W, wl, rng):
    nel = wl.nup + (wl.ndn if wl.walker_type == COLLINEAR else 0)
    return (rng.standard_normal((W, nel * wl.M)) + 1j * rng.standard_normal((W, nel * wl.M))) / 4


@pytest.mark.parametrize("walker_type", [CLOSED, COLLINEAR])
def test_thc_matches_cholesky(walker_type):
    wl, X, Luv = make_thc_system(seed=3, M=12, N=4, nu=30, nv=20, walker_type=walker_type)
    ref = O.Real3IndexFactorization(wl.walker_type, wl.M, wl.nup, wl.ndn, wl.Likn, wl.hij,
                                    wl.E0, wl.PsiT)
    thc = T.THCOps(wl.walker_type, wl.M, wl.nup, wl.ndn, X, Luv, wl.hij, wl.E0, wl.PsiT)
    rng = np.random.default_rng(1)
    G = _G(5, wl, rng)
    dt = 0.01
    np.testing.assert_allclose(thc.vbias(G, dt), ref.vbias(G, dt), atol=1e-13, rtol=1e-11)
    x = rng.standard_normal((5, wl.Nc)) + 1j * rng.standard_normal((5, wl.Nc))
    np.testing.assert_allclose(thc.vHS(x, dt)[0], ref.vHS(x, dt)[0], atol=1e-13, rtol=1e-11)
    np.testing.assert_allclose(thc.energy(G), ref.energy(G), atol=1e-12, rtol=1e-11)
    np.testing.assert_allclose(thc.vexx[0], ref.vexx[0], atol=1e-13)
    vmf = rng.standard_normal(wl.Nc) * 0.1
    np.testing.assert_allclose(thc.getOneBodyPropagatorMatrix(dt, vmf),
                               ref.getOneBodyPropagatorMatrix(dt, vmf), atol=1e-13)


def test_cholesky_from_thc_is_symmetric():
    _, X, Luv = make_thc_system(seed=0, M=10, N=3, nu=20, nv=8)
    L = T.cholesky_from_thc(X, Luv)[0]
    assert np.max(np.abs(L - L.transpose(1, 0, 2))) == 0.0
