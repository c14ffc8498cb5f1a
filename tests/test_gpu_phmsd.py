"""PHMSD energy kernels through the C ABI on the GPU: the reference's golden values
(tests/test_phmsd_components.cpp:41-47) and the oracle at other sizes."""
import numpy as np
import pytest
import torch

from oracle import phmsd as P
from tests.golden import phmsd_golden as g
from tests.gpu_helpers import rel_err, to_dev, to_host

pytestmark = pytest.mark.gpu


def _i32(x, cuda):
    return torch.as_tensor(np.ascontiguousarray(x, dtype=np.int32), device=cuda)


def _run2(cuda, iexcit, refc, T, R, wgt, EX0=None, EJ0=None):
    from safire_b200 import afqmc as A
    nw, ndet, nex, nact = R.shape
    EX = to_dev(np.zeros(nw, complex) if EX0 is None else EX0)
    EJ = to_dev(np.zeros(nw, complex) if EJ0 is None else EJ0)
    KE = torch.zeros((ndet, nw, T.shape[2]), dtype=torch.complex128, device=cuda)
    A.phmsd.ph_excited_2body_energy(_i32(iexcit, cuda), _i32(refc, cuda), to_dev(T), to_dev(R),
                                    to_dev(wgt), EX, EJ, KE)
    return to_host(EX), to_host(EJ), to_host(KE)


@pytest.mark.parametrize("nex", [1, 2, 3, 4, 5])
def test_ph_excited_2body_golden(cuda, nex):
    iexcit, refc, T, R, wgt = g.fixture(nex)
    EX, EJ, _ = _run2(cuda, iexcit, refc, T, R, wgt)
    ref = g.EXJ_REF[nex - 1]
    assert abs(EX[0] - ref[0]) <= 1e-8 * abs(ref[0]), (EX[0], ref[0])
    assert abs(EJ[0] - ref[1]) <= 1e-8 * abs(ref[1]), (EJ[0], ref[1])


def _random_case(seed, nw, ndet, nex, nact, nelec, nchol):
    rs = np.random.default_rng(seed)
    rc = lambda *s: rs.standard_normal(s) + 1j * rs.standard_normal(s)  # noqa: E731
    refc = rs.permutation(nact)[:nelec].astype(np.int32)
    virt = np.setdiff1d(np.arange(nact), refc)
    iexcit = np.zeros((ndet, 2 * nex), dtype=np.int32)
    for d in range(ndet):
        iexcit[d, :nex] = rs.choice(nelec, nex, replace=False)
        iexcit[d, nex:] = rs.choice(virt, nex, replace=False)
    return iexcit, refc, rc(nw, nelec, nchol, nact), rc(nw, ndet, nex, nact), rc(ndet, nw)


@pytest.mark.parametrize("nex", [1, 2, 3, 4])
def test_ph_excited_2body_vs_oracle(cuda, nex):
    iexcit, refc, T, R, wgt = _random_case(10 + nex, 3, 37, nex, 23, 9, 70)
    rs = np.random.default_rng(99)
    EX0 = rs.standard_normal(3) + 1j * rs.standard_normal(3)
    EJ0 = rs.standard_normal(3) + 1j * rs.standard_normal(3)
    EX, EJ, KE = _run2(cuda, iexcit, refc, T, R, wgt, EX0, EJ0)
    EXo, EJo, KEo = P.ph_excited_2body_energy_dense_cholesky(iexcit, refc, T, R, wgt, EX0, EJ0)
    assert rel_err(EX, EXo) < 1e-10
    assert rel_err(EJ, EJo) < 1e-10
    assert rel_err(KE, KEo) < 1e-12


@pytest.mark.parametrize("nex", [1, 3])
def test_ph_excited_1body_vs_oracle(cuda, nex):
    from safire_b200 import afqmc as A
    iexcit, refc, T, R, wgt = _random_case(20 + nex, 4, 29, nex, 31, 11, 8)
    rs = np.random.default_rng(7)
    S = rs.standard_normal((4, 11, 31)) + 1j * rs.standard_normal((4, 11, 31))
    E0 = rs.standard_normal(4) + 1j * rs.standard_normal(4)
    E = to_dev(E0.copy())
    A.phmsd.ph_excited_1body_energy(_i32(iexcit, cuda), _i32(refc, cuda), to_dev(S), to_dev(R),
                                    to_dev(wgt), E)
    Eo = P.ph_excited_1body_energy(iexcit, refc, S, R, wgt, E0)
    assert rel_err(to_host(E), Eo) < 1e-12


def test_ph_excited_rejects_bad_index(cuda):
    """A hole outside the electron range is reported before any kernel reads with it."""
    from safire_b200 import afqmc as A
    from safire_b200.capi import AfqmcError
    iexcit, refc, T, R, wgt = _random_case(5, 1, 4, 2, 12, 5, 6)
    iexcit[2, 0] = 5  # nelec = 5
    with pytest.raises(AfqmcError):
        _run2(cuda, iexcit, refc, T, R, wgt)


def _trial(M, nup, ndn, nocc, nvirt, ndet, seed):
    from safire_b200.synth import make_hamiltonian, make_phmsd_trial
    h1, _ = make_hamiltonian(M, 2, 0.99, seed)
    _, C = np.linalg.eigh(h1)
    return make_phmsd_trial(M, nup, ndn, C, nocc=nocc, nvirt=nvirt, ndet=ndet, seed=seed)


@pytest.mark.parametrize("M,nup,ndn,nocc,nvirt,ndet,W", [(24, 6, 5, 4, 8, 120, 3),
                                                        (60, 15, 15, 8, 20, 700, 17)])
def test_phmsd_log_overlap_vs_oracle(cuda, M, nup, ndn, nocc, nvirt, ndet, W):
    """Woodbury log overlap of a multi-determinant trial (PHMSD.cpp:804-900) against the
    oracle, walker rows in the walker-buffer layout with extra property columns."""
    from safire_b200 import afqmc as A
    t = _trial(M, nup, ndn, nocc, nvirt, ndet, seed=M)
    rs = np.random.default_rng(M + 1)
    Su = (rs.standard_normal((W, M, nup)) + 1j * rs.standard_normal((W, M, nup))) / np.sqrt(M)
    Sd = (rs.standard_normal((W, M, ndn)) + 1j * rs.standard_normal((W, M, ndn))) / np.sqrt(M)
    row = np.concatenate([Su.reshape(W, -1), Sd.reshape(W, -1), np.zeros((W, 11))], axis=1)
    wbuf = to_dev(row)
    ov = torch.zeros(W, dtype=torch.complex128, device=cuda)
    A.PHMSD(t).Log_Overlap(wbuf, ov)
    ref, _ = P.phmsd_log_overlap(t, Su, Sd)
    got = to_host(ov)
    # the log's imaginary part is a phase: compare modulo 2 pi
    d = got - ref
    d = d.real + 1j * ((d.imag + np.pi) % (2 * np.pi) - np.pi)
    assert np.max(np.abs(d)) < 1e-10, (got, ref)


@pytest.mark.parametrize("mixed", [False, True], ids=["complex128", "mixed"])
@pytest.mark.parametrize("M,nup,ndn,Nc,nocc,nvirt,ndet,W,block", [
    (16, 4, 3, 6, 3, 5, 40, 3, 0), (40, 10, 9, 30, 6, 14, 300, 21, 8),
    # N * nact too large for the shared-memory tables: the per-shell R-row kernels
    (80, 40, 38, 8, 6, 30, 30, 3, 0)])
def test_phmsd_energy_vs_oracle(cuda, M, nup, ndn, Nc, nocc, nvirt, ndet, W, block, mixed):
    """PHMSD energy_alg1 on the GPU (walker blocks, excitation shells, spin couplings) against
    the oracle's restatement (itself pinned against single-determinant energies).  Complex128:
    1e-10.  Mixed precision (complex64 tables and per-determinant sums): 5e-5 relative on the
    energy components (single precision over sums of up to a few hundred terms per determinant
    and Cholesky vector, with the Woodbury inverses of the excitation blocks amplifying them;
    measured up to 1.7e-5), the overlaps still 1e-10 (complex128)."""
    from safire_b200 import afqmc as A
    from safire_b200.synth import make_hamiltonian, make_phmsd_trial
    h1, Likn = make_hamiltonian(M, Nc, 0.9, seed=M)
    _, C = np.linalg.eigh(h1)
    t = make_phmsd_trial(M, nup, ndn, C, nocc=nocc, nvirt=nvirt, ndet=ndet, seed=M)
    hij = h1[None].astype(complex)
    rs = np.random.default_rng(M + 2)
    Su = (rs.standard_normal((W, M, nup)) + 1j * rs.standard_normal((W, M, nup))) / np.sqrt(M)
    Sd = (rs.standard_normal((W, M, ndn)) + 1j * rs.standard_normal((W, M, ndn))) / np.sqrt(M)
    wbuf = to_dev(np.concatenate([Su.reshape(W, -1), Sd.reshape(W, -1), np.zeros((W, 11))], 1))
    ph = A.PHMSD(t)
    ph.set_hamiltonian(Likn[None], hij, 0.3)
    if mixed:
        ph.set_precision(A.PREC_MIXED)
    E = torch.zeros((W, 3), dtype=torch.complex128, device=cuda)
    ov = torch.zeros(W, dtype=torch.complex128, device=cuda)
    ph.Energy(wbuf, E, ov, block=block)
    H = P.ActiveSpaceHamiltonian(t, Likn[None], hij, 0.3)
    Eo, ovo = P.phmsd_energy(t, H, Su, Sd)
    errs = [rel_err(to_host(E)[:, q], Eo[:, q]) for q in range(3)]
    print(f"PHMSD energy ({'mixed' if mixed else 'complex128'}) E1/EXX/EJ rel errs",
          ["%.2e" % e for e in errs])
    assert max(errs) < (5e-5 if mixed else 1e-10)
    d = to_host(ov) - ovo
    d = d.real + 1j * ((d.imag + np.pi) % (2 * np.pi) - np.pi)
    assert np.max(np.abs(d)) < 1e-10


@pytest.mark.gpu
@pytest.mark.parametrize("M,nup,ndn,Nc,nocc,nvirt,ndet,W,block", [
    (24, 5, 4, 30, 5, 8, 40, 5, 0),
    (40, 9, 9, 64, 9, 14, 300, 7, 3),
    (64, 12, 10, 48, 12, 20, 800, 33, 0),
])
def test_phmsd_density_matrix_and_vbias_vs_oracle(cuda, M, nup, ndn, Nc, nocc, nvirt, ndet, W,
                                                   block):
    """PHMSD MixedDensityMatrix (full Woodbury R per electron, then R^T G_ref / Ov) and the
    active-space vbias on the GPU against the oracle (whose density matrix is pinned against the
    determinant-by-determinant sum)."""
    from safire_b200 import afqmc as A
    from safire_b200.synth import make_hamiltonian, make_phmsd_trial
    h1, Likn = make_hamiltonian(M, Nc, 0.9, seed=M + 5)
    _, C = np.linalg.eigh(h1)
    t = make_phmsd_trial(M, nup, ndn, C, nocc=nocc, nvirt=nvirt, ndet=ndet, seed=M + 1)
    hij = h1[None].astype(complex)
    rs = np.random.default_rng(M + 3)
    Su = (rs.standard_normal((W, M, nup)) + 1j * rs.standard_normal((W, M, nup))) / np.sqrt(M)
    Sd = (rs.standard_normal((W, M, ndn)) + 1j * rs.standard_normal((W, M, ndn))) / np.sqrt(M)
    wbuf = to_dev(np.concatenate([Su.reshape(W, -1), Sd.reshape(W, -1), np.zeros((W, 7))], 1))
    ph = A.PHMSD(t)
    ph.set_hamiltonian(Likn[None], hij, 0.0)
    na = t.orbmat[0].shape[0] + t.orbmat[1].shape[0]
    G = torch.zeros((W, na, M), dtype=torch.complex128, device=cuda)
    ov = torch.zeros(W, dtype=torch.complex128, device=cuda)
    ph.MixedDensityMatrix(wbuf, G, ov, block=block)
    Go, ovo = P.phmsd_mixed_density_matrix(t, Su, Sd)
    assert rel_err(to_host(G), Go) < 1e-10
    d = to_host(ov) - ovo
    d = d.real + 1j * ((d.imag + np.pi) % (2 * np.pi) - np.pi)
    assert np.max(np.abs(d)) < 1e-10
    v = torch.zeros((W, Nc), dtype=torch.complex128, device=cuda)
    ph.vbias(G, v, 0.005)
    H = P.ActiveSpaceHamiltonian(t, Likn[None], hij, 0.0)
    vo = P.phmsd_vbias(H, Go, 0.005, t.orbmat[0].shape[0])
    assert rel_err(to_host(v), vo) < 1e-10


@pytest.mark.parametrize("W,steps,mixed", [(6, 4, False), (6, 4, True)],
                         ids=["complex128", "mixed"])
def test_phmsd_propagation_steps_vs_oracle(cuda, W, steps, mixed):
    """Walker steps with a PHMSD trial attached to the propagator (PHMSD vbias and overlaps,
    COLLINEAR vHS and propagation, hybrid weight update, orthogonalisation) against the oracle's
    propagator driving the same PHMSD restatement, with the same field uniforms.  Complex128:
    1e-10.  Mixed precision (the vHS and the Taylor series of both spin blocks on the tensor
    cores, the trial's vbias and overlaps in complex128): the walkers and weights within 1e-4,
    the log-overlaps within 1e-4 absolute (9 electrons), the fields' vbias exact as long as the
    walkers are the same (first step) and within 1e-4 after."""
    from oracle import afqmc as O
    from safire_b200 import afqmc as A
    from safire_b200 import capi
    from safire_b200.synth import make_hamiltonian, make_phmsd_trial
    M, nup, ndn, Nc, dt = 24, 5, 4, 40, 0.01
    h1, Likn = make_hamiltonian(M, Nc, 0.9, seed=7)
    _, C = np.linalg.eigh(h1)
    t = make_phmsd_trial(M, nup, ndn, C, nocc=4, nvirt=8, ndet=60, seed=3)
    hij = h1[None].astype(complex)
    PsiT = [t.orbmat[0][t.refc[0]], t.orbmat[1][t.refc[1]]]
    ham = A.HamiltonianOperations(A.COLLINEAR, M, nup, ndn, Likn[None], hij, 0.2, PsiT)
    oham = O.Real3IndexFactorization(O.COLLINEAR, M, nup, ndn, Likn[None], hij, 0.2, PsiT)
    vMF = O.NOMSD(oham, PsiT).vMF(dt) * 0.8  # any mean field: both sides take it as given
    ph = A.PHMSD(t)
    ph.set_hamiltonian(Likn[None], hij, 0.2)
    prec = A.PREC_MIXED if mixed else A.PREC_FP64
    tol, tol_ov = (1e-4, 1e-4) if mixed else (1e-10, 1e-9)
    prop = A.Propagator(ham, A.default_params(dt=dt, precision=prec), W)
    prop.set_trial(ph, vMF)
    wset = A.WalkerSet(A.COLLINEAR, M, nup, ndn, W)
    wset.init_from_trial(ham)
    ov = torch.zeros(W, dtype=torch.complex128, device=cuda)
    ph.Log_Overlap(wset.buffer, ov)
    wset.setProperty(capi.OVLP, to_host(ov))
    torch.cuda.synchronize()

    owfn = P.PHMSDWavefunction(t, oham, Likn[None], hij, vMF)
    oprop = O.Propagator(owfn, O.PropagatorParams(dt=dt))
    P1d, vMFd = prop.P1_vMF()
    assert rel_err(P1d, oprop.P1) < 1e-12 and rel_err(vMFd, oprop.vMF) < 1e-14
    ows = O.WalkerSet(to_host(wset.SlaterMatrices(0)).copy(), to_host(wset.SlaterMatrices(1)).copy(),
                      to_host(wset.properties()).copy(), W, O.COLLINEAR)
    assert np.max(np.abs(ows.props[:, O.OVLP] - owfn.Log_Overlap(ows.SA, ows.SB))) < 1e-10
    Eshift = -1.3
    rs = np.random.default_rng(5)
    for step in range(steps):
        u = rs.random((W, Nc))
        prop.Propagate(wset, Eshift, to_dev(u, torch.float64))
        last = prop.last_step(W)
        oprop.propagate(ows, Eshift, u)
        lo = oprop.last
        tv = 1e-10 if (step == 0 or not mixed) else tol
        assert rel_err(to_host(last.vbias), lo["vbias"]) < tv, step
        assert rel_err(to_host(last.X), lo["X"]) < tv, step
        d = to_host(last.new_ovlp) - lo["new_ov"]
        assert np.max(np.abs(d.real + 1j * ((d.imag + np.pi) % (2 * np.pi) - np.pi))) < tol_ov, step
        assert rel_err(to_host(wset.SlaterMatrices(0)), ows.SA) < tol, step
        assert rel_err(to_host(wset.SlaterMatrices(1)), ows.SB) < tol, step
        props = to_host(wset.properties())
        assert rel_err(props[:, O.WEIGHT], ows.props[:, O.WEIGHT]) < tol, step
        if step == 1:
            prop.Orthogonalize(wset)
            oprop.orthogonalize(ows)
            assert rel_err(to_host(wset.SlaterMatrices(1)), ows.SB) < tol
            d = to_host(wset.properties())[:, O.OVLP] - ows.props[:, O.OVLP]
            assert np.max(np.abs(d.real + 1j * ((d.imag + np.pi) % (2 * np.pi) - np.pi))) < tol_ov
    assert ham.device_error_flag() == 0
    prop.set_trial(None)
