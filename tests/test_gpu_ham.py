"""HamiltonianOperations (Real3IndexFactorization) through the C ABI vs the oracle."""
import numpy as np
import pytest
import torch

from oracle import afqmc as O
from safire_b200.synth import make_workload
from tests.gpu_helpers import make_pair, rand_c, rel_err, to_dev, to_host

pytestmark = pytest.mark.gpu
TOL = 1e-10


@pytest.fixture(scope="module")
def cfg1(cuda):
    wl = make_workload("cfg1", W=16)
    dham, oham, owfn = make_pair(wl)
    return wl, dham, oham, owfn


def test_tensors(cfg1):
    wl, dham, oham, _ = cfg1
    t = dham.tensors()
    assert rel_err(t.Lnak[0], oham.Lnak[0]) < TOL
    assert rel_err(t.haj, oham.haj) < TOL
    assert rel_err(t.vexx, oham.vexx) < TOL


def test_vbias(cfg1):
    wl, dham, oham, _ = cfg1
    rs = np.random.default_rng(1)
    G = rand_c(rs, wl.W, wl.nup * wl.M)
    v = torch.zeros((wl.W, wl.Nc), dtype=torch.complex128, device="cuda")
    dham.vbias(to_dev(G), v, wl.dt)
    assert rel_err(to_host(v), oham.vbias(G, wl.dt)) < TOL


def test_vhs(cfg1):
    wl, dham, oham, _ = cfg1
    rs = np.random.default_rng(2)
    X = rand_c(rs, wl.W, wl.Nc)
    V = dham.vHS(to_dev(X), wl.dt)
    assert rel_err(to_host(V), oham.vHS(X, wl.dt)) < TOL


def test_energy(cfg1):
    wl, dham, oham, _ = cfg1
    rs = np.random.default_rng(3)
    G = rand_c(rs, wl.W, wl.nup * wl.M, scale=0.2)
    E = torch.zeros((wl.W, 3), dtype=torch.complex128, device="cuda")
    dham.energy(E, to_dev(G))
    Eo = oham.energy(G)
    for q in range(3):
        assert rel_err(to_host(E)[:, q], Eo[:, q]) < TOL
    # partial energies
    dham.energy(E, to_dev(G), addH1=False, addEJ=False, addEXX=True)
    Eo = oham.energy(G, addH1=False, addEJ=False, addEXX=True)
    assert rel_err(to_host(E), Eo) < TOL


def test_energy_real_and_complex_trial(cuda):
    """A complex trial takes the complex Lnak path (no real-trial specialisation)."""
    wl = make_workload("cfg1", W=5, M=16, N=4, Nc=24)
    rs = np.random.default_rng(9)
    wl.PsiT = [wl.PsiT[0] * np.exp(1j * rs.random((4, 1)))]
    dham, oham, _ = make_pair(wl)
    G = rand_c(rs, 5, 4 * 16, scale=0.3)
    E = torch.zeros((5, 3), dtype=torch.complex128, device="cuda")
    dham.energy(E, to_dev(G))
    assert rel_err(to_host(E), oham.energy(G)) < TOL
    v = torch.zeros((5, 24), dtype=torch.complex128, device="cuda")
    dham.vbias(to_dev(G), v, 0.01)
    assert rel_err(to_host(v), oham.vbias(G, 0.01)) < TOL


def test_vmf_and_one_body(cfg1):
    wl, dham, oham, owfn = cfg1
    from safire_b200 import afqmc as A
    dwfn = A.NOMSD(dham)
    vmf = dwfn.vMF(wl.dt)
    vmf_o = owfn.vMF(wl.dt)
    assert rel_err(vmf, vmf_o) < TOL
    vm = vmf_o.real.astype(complex)
    H1 = dham.getOneBodyPropagatorMatrix(wl.dt, vm)
    assert rel_err(H1, oham.getOneBodyPropagatorMatrix(wl.dt, vm)) < TOL


@pytest.mark.parametrize("denseP1", [0, 1])
def test_generate_p1(cfg1, denseP1):
    wl, dham, oham, owfn = cfg1
    from safire_b200 import afqmc as A
    prop = A.Propagator(dham, A.default_params(dt=wl.dt, denseP1=denseP1), wl.W)
    P1, vMF = prop.P1_vMF()
    P1o, vMFo = O.generateP1(owfn, wl.dt, bool(denseP1))
    assert rel_err(vMF, vMFo) < TOL
    assert rel_err(P1, P1o) < TOL
    # the truncation keeps the same sparsity pattern (|x| > 1e-8)
    assert np.array_equal(P1 != 0, P1o != 0)


def test_bad_arguments_raise(cfg1):
    wl, dham, _, _ = cfg1
    from safire_b200.capi import AfqmcError
    from safire_b200 import capi
    with pytest.raises(AfqmcError):
        capi.call("afqmc_ham_energy", dham.handle, None, None, 4, 1, 1, 1, 0, None)
    with pytest.raises(AfqmcError):
        # addEJ without addEXX is rejected as in the reference
        E = torch.zeros((2, 3), dtype=torch.complex128, device="cuda")
        G = torch.zeros((2, wl.nup * wl.M), dtype=torch.complex128, device="cuda")
        dham.energy(E, G, addH1=True, addEJ=True, addEXX=False)
