"""NOMSD with several determinants through the C ABI against the oracle: log overlap, energy,
the combined full density matrix, the full-G vbias, and propagation steps with the trial
attached (CLOSED and COLLINEAR)."""
import numpy as np
import pytest
import torch

from oracle import afqmc as O
from safire_b200.synth import make_hamiltonian
from tests.gpu_helpers import rel_err, to_dev, to_host

pytestmark = pytest.mark.gpu


def _wrap(d):
    return d.real + 1j * ((d.imag + np.pi) % (2 * np.pi) - np.pi)


def _setup(wt, nup, ndn, M=14, Nc=12, W=5):
    from safire_b200 import afqmc as A
    h1, Likn = make_hamiltonian(M, Nc, 0.9, seed=4)
    _, C = np.linalg.eigh(h1)
    rs = np.random.default_rng(wt)
    occs = [list(range(nup)), list(range(nup - 1)) + [nup], list(range(nup - 2)) + [nup, nup + 1]]
    PsiTs = []
    for occ in occs:
        P = [np.ascontiguousarray(C[:, occ].T).astype(complex)]
        if wt == A.COLLINEAR:
            P.append(np.ascontiguousarray(C[:, list(range(ndn - 1)) + [ndn + 1]].T).astype(complex))
        PsiTs.append(P)
    ci = np.array([0.9, 0.3 + 0.1j, -0.25])
    hij = h1[None].astype(complex)
    hams = [A.HamiltonianOperations(wt, M, nup, ndn, Likn[None], hij, 0.1, P) for P in PsiTs]
    ohams = [O.Real3IndexFactorization(wt, M, nup, ndn, Likn[None], hij, 0.1, P) for P in PsiTs]
    SA = rs.standard_normal((W, M, nup)) + 1j * rs.standard_normal((W, M, nup))
    SB = rs.standard_normal((W, M, ndn)) + 1j * rs.standard_normal((W, M, ndn)) \
        if wt == A.COLLINEAR else None
    return A, hams, ohams, PsiTs, ci, SA, SB, Likn, hij, M, Nc, W


@pytest.mark.parametrize("wt,nup,ndn", [(1, 4, 4), (2, 4, 3)])
def test_multidet_overlap_energy_density_vbias(cuda, wt, nup, ndn):
    A, hams, ohams, PsiTs, ci, SA, SB, Likn, hij, M, Nc, W = _setup(wt, nup, ndn)
    md = A.NOMSDMulti(hams, ci)
    omd = O.NOMSDMulti(ohams, PsiTs, ci)
    wset = A.WalkerSet(wt, M, nup, ndn, W)
    wset.init_from_trial(hams[0])
    wset.SlaterMatrices(0).copy_(to_dev(SA))
    if SB is not None:
        wset.SlaterMatrices(1).copy_(to_dev(SB))
    lo = md.Log_Overlap(wset)
    lo_o = omd.Log_Overlap(SA, SB)
    assert np.max(np.abs(_wrap(to_host(lo) - lo_o))) < 1e-10
    E, ov = md.Energy(wset, set_properties=True)
    Eo, ovo = omd.Energy(SA, SB)
    assert rel_err(to_host(E), Eo) < 1e-10
    assert np.max(np.abs(_wrap(to_host(ov) - ovo))) < 1e-10
    # the density matrix weighs the determinants relative to the walkers' OVLP property
    log_m = to_host(wset.properties()[:, A.capi.OVLP])
    G, ovG = md.MixedDensityMatrix(wset)
    Go, ovGo = omd.MixedDensityMatrix(SA, SB, log_m)
    assert rel_err(to_host(G), Go) < 1e-10
    assert rel_err(to_host(ovG), ovGo) < 1e-10
    v = torch.empty((W, Nc), dtype=torch.complex128, device=cuda)
    md.vbias(G, v, 0.01)
    assert rel_err(to_host(v), omd.vbias(SA, SB, 0.01)) < 1e-10


@pytest.mark.parametrize("wt,nup,ndn", [(1, 4, 4), (2, 4, 3)])
def test_multidet_propagation_vs_oracle(cuda, wt, nup, ndn):
    A, hams, ohams, PsiTs, ci, SA, SB, Likn, hij, M, Nc, W = _setup(wt, nup, ndn)
    dt = 0.01
    md = A.NOMSDMulti(hams, ci)
    vMF = O.NOMSD(ohams[0], PsiTs[0]).vMF(dt) * 0.7  # any mean field: both sides take it
    omd = O.NOMSDMulti(ohams, PsiTs, ci, vMF)
    prop = A.Propagator(hams[0], A.default_params(dt=dt), W)
    prop.set_trial(md, vMF)
    wset = A.WalkerSet(wt, M, nup, ndn, W)
    wset.init_from_trial(hams[0])
    wset.SlaterMatrices(0).copy_(to_dev(SA))
    if SB is not None:
        wset.SlaterMatrices(1).copy_(to_dev(SB))
    wset.setProperty(A.capi.OVLP, to_host(md.Log_Overlap(wset)))
    torch.cuda.synchronize()
    oprop = O.Propagator(omd, O.PropagatorParams(dt=dt))
    P1d, vMFd = prop.P1_vMF()
    assert rel_err(P1d, oprop.P1) < 1e-12
    ows = O.WalkerSet(SA.copy(), None if SB is None else SB.copy(),
                      to_host(wset.properties()).copy(), W, wt)
    rs = np.random.default_rng(8)
    for step in range(3):
        u = rs.random((W, Nc))
        prop.Propagate(wset, -1.0, to_dev(u, torch.float64))
        last = prop.last_step(W)
        oprop.propagate(ows, -1.0, u)
        assert rel_err(to_host(last.vbias), oprop.last["vbias"]) < 1e-10, step
        assert np.max(np.abs(_wrap(to_host(last.new_ovlp) - oprop.last["new_ov"]))) < 1e-9, step
        assert rel_err(to_host(wset.SlaterMatrices(0)), ows.SA) < 1e-10, step
        props = to_host(wset.properties())
        assert rel_err(props[:, O.WEIGHT], ows.props[:, O.WEIGHT]) < 1e-10, step
    prop.Orthogonalize(wset)
    oprop.orthogonalize(ows)
    d = to_host(wset.properties())[:, O.OVLP] - ows.props[:, O.OVLP]
    assert np.max(np.abs(_wrap(d))) < 1e-9
    prop.set_trial(None)


@pytest.mark.parametrize("wt,nup,ndn", [(1, 2, 2), (2, 2, 2)])
def test_multidet_batched_walker_chunks(cuda, wt, nup, ndn):
    """300 determinants: the batched step goes over the walkers in chunks of 65535 // 300 = 218
    (a bound on the batched launches' grids), so 230 walkers take a full and a ragged chunk."""
    from safire_b200 import afqmc as A
    M, Nc, W, nd = 8, 6, 230, 300
    h1, Likn = make_hamiltonian(M, Nc, 0.9, seed=5)
    _, C = np.linalg.eigh(h1)
    rs = np.random.default_rng(11)
    PsiTs = []
    for _ in range(nd):
        P = [np.ascontiguousarray(C[:, np.sort(rs.choice(M, nup, replace=False))].T).astype(complex)]
        if wt == A.COLLINEAR:
            P.append(np.ascontiguousarray(
                C[:, np.sort(rs.choice(M, ndn, replace=False))].T).astype(complex))
        PsiTs.append(P)
    ci = rs.standard_normal(nd) + 1j * rs.standard_normal(nd)
    hij = h1[None].astype(complex)
    hams = [A.HamiltonianOperations(wt, M, nup, ndn, Likn[None], hij, 0.1, P) for P in PsiTs]
    ohams = [O.Real3IndexFactorization(wt, M, nup, ndn, Likn[None], hij, 0.1, P)
             for P in PsiTs[:1]] * nd
    md = A.NOMSDMulti(hams, ci)
    omd = O.NOMSDMulti(ohams, PsiTs, ci)
    SA = rs.standard_normal((W, M, nup)) + 1j * rs.standard_normal((W, M, nup))
    SB = rs.standard_normal((W, M, ndn)) + 1j * rs.standard_normal((W, M, ndn)) \
        if wt == A.COLLINEAR else None
    wset = A.WalkerSet(wt, M, nup, ndn, W)
    wset.init_from_trial(hams[0])
    wset.SlaterMatrices(0).copy_(to_dev(SA))
    if SB is not None:
        wset.SlaterMatrices(1).copy_(to_dev(SB))
    lo_o = omd.Log_Overlap(SA, SB)
    lo = md.Log_Overlap(wset)
    assert np.max(np.abs(_wrap(to_host(lo) - lo_o))) < 1e-10
    wset.setProperty(A.capi.OVLP, lo_o)
    G, ovG = md.MixedDensityMatrix(wset)
    Go, ovGo = omd.MixedDensityMatrix(SA, SB, lo_o)
    assert rel_err(to_host(G), Go) < 1e-10
    assert rel_err(to_host(ovG), ovGo) < 1e-10
