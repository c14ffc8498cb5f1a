"""The MixedEstimator's OneRDM (single reference) through the C ABI against the oracle, for
CLOSED and COLLINEAR walkers with random Slater matrices and weights."""
import numpy as np
import pytest
import torch

from oracle import afqmc as O
from safire_b200.synth import make_hamiltonian
from tests.gpu_helpers import rel_err, to_dev, to_host

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("wt,nup,ndn", [(1, 6, 6), (2, 5, 3)])
def test_onerdm_vs_oracle(cuda, wt, nup, ndn):
    from safire_b200 import afqmc as A
    from safire_b200 import capi
    M, Nc, W = 20, 24, 9
    h1, Likn = make_hamiltonian(M, Nc, 0.9, seed=3)
    _, C = np.linalg.eigh(h1)
    PsiT = [np.ascontiguousarray(C[:, :nup].T).astype(complex)]
    if wt == A.COLLINEAR:
        PsiT.append(np.ascontiguousarray(C[:, 1:ndn + 1].T).astype(complex))
    hij = h1[None].astype(complex)
    ham = A.HamiltonianOperations(wt, M, nup, ndn, Likn[None], hij, 0.0, PsiT)
    wset = A.WalkerSet(wt, M, nup, ndn, W)
    wset.init_from_trial(ham)
    rs = np.random.default_rng(wt)
    SA = rs.standard_normal((W, M, nup)) + 1j * rs.standard_normal((W, M, nup))
    wset.SlaterMatrices(0).copy_(to_dev(SA))
    SB = None
    if wt == A.COLLINEAR:
        SB = rs.standard_normal((W, M, ndn)) + 1j * rs.standard_normal((W, M, ndn))
        wset.SlaterMatrices(1).copy_(to_dev(SB))
    w = rs.random(W) + 0.2 + 0.1j * rs.standard_normal(W)
    wset.setProperty(capi.WEIGHT, w)
    torch.cuda.synchronize()
    rdm, wsum = A.NOMSD(ham).OneRDM(wset)
    oham = O.Real3IndexFactorization(wt, M, nup, ndn, Likn[None], hij, 0.0, PsiT)
    owfn = O.NOMSD(oham, PsiT)
    props = np.zeros((W, O.NPROP), complex)
    props[:, O.WEIGHT] = w
    ows = O.WalkerSet(SA, SB, props, W, wt)
    ref = O.onerdm(owfn, ows)
    assert rdm.shape == ref.shape
    assert rel_err(to_host(rdm), ref) < 1e-10
    assert abs(complex(wsum.item()) - w.sum()) < 1e-12 * abs(w.sum())
