"""THC HamiltonianOperations (THCOps) on the GPU through the C ABI: against the oracle's THC
restatement, against the library's own Cholesky path on the Cholesky vectors the THC factors
stand for, and a walker trajectory stepped with each."""
import numpy as np
import pytest
import torch

from oracle import thc as T
from safire_b200 import afqmc as A
from safire_b200 import capi
from safire_b200.driver import RunParams, Simulation
from safire_b200.synth import CLOSED, COLLINEAR, make_thc_system
from tests.gpu_helpers import rand_c, rel_err, to_dev, to_host

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _system(walker_type, W=9):
    wl, X, Luv = make_thc_system(seed=5, M=20, N=5, nu=48, nv=36, W=W, walker_type=walker_type)
    dthc = A.HamiltonianOperations.thc(wl.walker_type, wl.M, wl.nup, wl.ndn, X, Luv, wl.hij,
                                       wl.E0, wl.PsiT)
    othc = T.THCOps(wl.walker_type, wl.M, wl.nup, wl.ndn, X, Luv, wl.hij, wl.E0, wl.PsiT)
    return wl, X, Luv, dthc, othc


@pytest.mark.parametrize("walker_type", [CLOSED, COLLINEAR])
def test_thc_ops_vs_oracle(cuda, walker_type):
    wl, X, Luv, dthc, othc = _system(walker_type)
    rs = np.random.default_rng(2)
    nel = wl.nup + (wl.ndn if walker_type == COLLINEAR else 0)
    G = rand_c(rs, wl.W, nel * wl.M, scale=0.3)
    v = torch.zeros((wl.W, wl.Nc), dtype=torch.complex128, device="cuda")
    dthc.vbias(to_dev(G), v, wl.dt)
    assert rel_err(to_host(v), othc.vbias(G, wl.dt)) < TOL
    x = rand_c(rs, wl.W, wl.Nc)
    V = dthc.vHS(to_dev(x), wl.dt)
    assert rel_err(to_host(V), othc.vHS(x, wl.dt)) < TOL
    E = torch.zeros((wl.W, 3), dtype=torch.complex128, device="cuda")
    dthc.energy(E, to_dev(G))
    Eo = othc.energy(G)
    errs = [rel_err(to_host(E)[:, q], Eo[:, q]) for q in range(3)]
    print(f"THC vs oracle ({walker_type}): E1/EXX/EJ {['%.1e' % e for e in errs]}")
    assert max(errs) < TOL
    # (the ABI rejects addEJ without addEXX, as for the Cholesky form)
    for flags in [(False, False, True), (True, False, False), (False, True, True)]:
        dthc.energy(E, to_dev(G), *flags)
        assert rel_err(to_host(E), othc.energy(G, *flags)) < TOL
    vmf = rs.standard_normal(wl.Nc) * 0.05
    assert rel_err(dthc.getOneBodyPropagatorMatrix(wl.dt, vmf),
                   othc.getOneBodyPropagatorMatrix(wl.dt, vmf)) < TOL


@pytest.mark.parametrize("walker_type", [CLOSED, COLLINEAR])
def test_thc_vs_cholesky_on_device(cuda, walker_type):
    """The same Hamiltonian in both factorisations: the library's THC and Cholesky paths agree."""
    wl, X, Luv, dthc, _ = _system(walker_type)
    dchol = A.HamiltonianOperations(wl.walker_type, wl.M, wl.nup, wl.ndn, wl.Likn, wl.hij, wl.E0,
                                    wl.PsiT)
    rs = np.random.default_rng(4)
    nel = wl.nup + (wl.ndn if walker_type == COLLINEAR else 0)
    G = to_dev(rand_c(rs, wl.W, nel * wl.M, scale=0.3))
    v1 = torch.zeros((wl.W, wl.Nc), dtype=torch.complex128, device="cuda")
    v2 = torch.zeros_like(v1)
    dthc.vbias(G, v1, wl.dt)
    dchol.vbias(G, v2, wl.dt)
    assert rel_err(to_host(v1), to_host(v2)) < TOL
    E1 = torch.zeros((wl.W, 3), dtype=torch.complex128, device="cuda")
    E2 = torch.zeros_like(E1)
    dthc.energy(E1, G)
    dchol.energy(E2, G)
    assert rel_err(to_host(E1), to_host(E2)) < TOL


@pytest.mark.parametrize("walker_type", [CLOSED, COLLINEAR])
def test_thc_trajectory_matches_cholesky(cuda, walker_type):
    """Twelve steps (orthogonalisation every 5, comb every 5, energy every 4) from the same seeds
    with the THC and with the Cholesky operations: the walkers and the energies agree."""
    wl, X, Luv, dthc, _ = _system(walker_type, W=16)
    rp = RunParams(equilibration_steps=0, seed=11, walker_ortho_interval=5,
                   population_control_interval=5)
    sims = [Simulation.from_workload(wl, W=16, rp=rp, ham=dthc),
            Simulation.from_workload(wl, W=16, rp=rp)]
    es = [[], []]
    for step in range(12):
        for k, sim in enumerate(sims):
            sim.step(measure=False)
            if step % 4 == 3:
                es[k].append(sim.measure()[0])
    torch.cuda.synchronize()
    b0 = sims[0].wset.buffer.cpu().numpy()
    b1 = sims[1].wset.buffer.cpu().numpy()
    err = rel_err(b0, b1)
    print(f"THC vs Cholesky trajectory ({walker_type}): walkers {err:.1e}, energies "
          f"{np.max(np.abs(np.array(es[0]) - np.array(es[1]))):.1e}")
    assert err < 1e-8
    assert np.max(np.abs(np.array(es[0]) - np.array(es[1]))) < 1e-8


def test_thc_refuses_mixed_precision(cuda):
    wl, X, Luv, dthc, _ = _system(CLOSED)
    G = to_dev(np.zeros((wl.W, wl.nup * wl.M), dtype=np.complex128))
    E = torch.zeros((wl.W, 3), dtype=torch.complex128, device="cuda")
    with pytest.raises(capi.AfqmcError) as ex:
        dthc.energy(E, G, precision=A.PREC_MIXED)
    assert ex.value.status == capi.ERR_UNSUPPORTED
