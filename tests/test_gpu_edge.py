"""Edge cases the reference's code paths allow: calls on zero walkers (no work, outputs
untouched) and a COLLINEAR walker set with an empty spin sector (the reference returns early for
N = 0, density_matrix.hpp:561-567), stepped against the oracle."""
import numpy as np
import pytest
import torch

from oracle import afqmc as O
from safire_b200.synth import make_hamiltonian, make_workload
from tests.gpu_helpers import rel_err, to_dev, to_host

pytestmark = pytest.mark.gpu


def test_zero_walkers_are_no_ops(cuda):
    from safire_b200 import afqmc as A
    M, N, Nc = 10, 3, 6
    h1, Likn = make_hamiltonian(M, Nc, 0.9, seed=0)
    _, C = np.linalg.eigh(h1)
    PsiT = [np.ascontiguousarray(C[:, :N].T).astype(complex)]
    ham = A.HamiltonianOperations(A.CLOSED, M, N, N, Likn[None], h1[None].astype(complex), 0.0,
                                  PsiT)
    P = to_dev(PsiT[0])
    S = torch.zeros((0, M, N), dtype=torch.complex128, device=cuda)
    ov = torch.full((0,), 7 + 0j, dtype=torch.complex128, device=cuda)
    G = torch.zeros((0, N * M), dtype=torch.complex128, device=cuda)
    A.det_ops.Log_Overlap(P, S, ov)
    A.det_ops.MixedDensityMatrix(P, S, G, ov)
    A.det_ops.orthogonalize(S, ov)
    v = torch.zeros((0, Nc), dtype=torch.complex128, device=cuda)
    for prec in (A.PREC_FP64, A.PREC_MIXED):
        ham.vbias(G, v, 0.01, precision=prec)
        E = torch.zeros((0, 3), dtype=torch.complex128, device=cuda)
        ham.energy(E, G, precision=prec)
    torch.cuda.synchronize()


def test_empty_spin_sector_steps_vs_oracle(cuda):
    """COLLINEAR walkers with N_dn = 0: overlaps, energies and propagation steps (with
    orthogonalisation) match the oracle."""
    from safire_b200 import afqmc as A
    M, Nc, nup, ndn, W, dt = 12, 10, 4, 0, 5, 0.01
    h1, Likn = make_hamiltonian(M, Nc, 0.9, seed=1)
    _, C = np.linalg.eigh(h1)
    PsiT = [np.ascontiguousarray(C[:, :nup].T).astype(complex), np.zeros((0, M), complex)]
    hij = h1[None].astype(complex)
    ham = A.HamiltonianOperations(A.COLLINEAR, M, nup, ndn, Likn[None], hij, 0.0, PsiT)
    wset = A.WalkerSet(A.COLLINEAR, M, nup, ndn, W)
    wset.init_from_trial(ham)
    rs = np.random.default_rng(2)
    SA = rs.standard_normal((W, M, nup)) + 1j * rs.standard_normal((W, M, nup))
    wset.SlaterMatrices(0).copy_(to_dev(SA))
    wfn = A.NOMSD(ham)
    E, ov = wfn.Energy(wset, set_properties=True)
    oham = O.Real3IndexFactorization(O.COLLINEAR, M, nup, ndn, Likn[None], hij, 0.0, PsiT)
    owfn = O.NOMSD(oham, PsiT)
    SB = np.zeros((W, M, 0), complex)
    Eo, ovo = owfn.Energy(SA, SB)
    assert rel_err(to_host(E), Eo) < 1e-10
    d = to_host(ov) - ovo
    assert np.max(np.abs(d.real + 1j * ((d.imag + np.pi) % (2 * np.pi) - np.pi))) < 1e-10
    prop = A.Propagator(ham, A.default_params(dt=dt), W)
    oprop = O.Propagator(owfn, O.PropagatorParams(dt=dt))
    ows = O.WalkerSet(SA.copy(), SB.copy(), to_host(wset.properties()).copy(), W, O.COLLINEAR)
    for step in range(3):
        u = rs.random((W, Nc))
        prop.Propagate(wset, -1.0, to_dev(u, torch.float64))
        oprop.propagate(ows, -1.0, u)
        assert rel_err(to_host(wset.SlaterMatrices(0)), ows.SA) < 1e-10, step
        props = to_host(wset.properties())
        assert rel_err(props[:, O.WEIGHT], ows.props[:, O.WEIGHT]) < 1e-10, step
    prop.Orthogonalize(wset)
    oprop.orthogonalize(ows)
    assert rel_err(to_host(wset.SlaterMatrices(0)), ows.SA) < 1e-10


def test_bounded_wait_times_out(cuda):
    """A bounded device wait that nothing completes gives up after its budget (about 0.05 s
    here), reports AFQMC_ERR_TIMEOUT and sets bit 0 of the Hamiltonian's error word, and the
    context stays usable: a mixed-precision contraction right after it runs and matches the
    oracle, and clearing the word leaves it at zero."""
    from safire_b200 import afqmc as A
    from safire_b200 import capi
    from tests.gpu_helpers import make_pair, rand_c

    wl = make_workload("cfg1", W=16)
    dham, oham, _ = make_pair(wl)
    dham.clear_device_error()
    assert dham.device_error_flag() == 0
    with pytest.raises(capi.AfqmcError) as ei:
        dham.wait_selftest(100_000_000)
    assert ei.value.status == capi.ERR_TIMEOUT
    assert dham.device_error_flag() & 1
    dham.clear_device_error()
    assert dham.device_error_flag() == 0
    rs = np.random.default_rng(9)
    G = rand_c(rs, wl.W, wl.nup * wl.M, scale=0.3)
    v = torch.zeros((wl.W, wl.Nc), dtype=torch.complex128, device="cuda")
    dham.vbias(to_dev(G), v, wl.dt, precision=A.PREC_MIXED)
    assert rel_err(to_host(v), oham.vbias(G, wl.dt)) < 2e-5
    assert dham.device_error_flag() == 0
