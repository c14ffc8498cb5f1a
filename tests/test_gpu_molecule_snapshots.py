"""The CUDA path against the reference's own seeded runs: every snapshot of its functional tests
that this library covers (BH, N2 and Li; one NOMSD determinant, 34 NOMSD determinants, PHMSD
over its reference orbitals and over a rotated complex reference; CLOSED and COLLINEAR walkers,
a spin-resolved one-body Hamiltonian, an empty beta sector) is
rerun through the C ABI with the reference's host random streams (Simulation.use_host_fields and
the comb's own stream).  The mixed-estimator energy, and for the single-determinant cases the
mixed and back-propagated one-body density matrices, match the reference's reported means
(over the whole number of bins its tools average; see tests/test_molecule_snapshots.py)."""
import numpy as np
import pytest
import torch

from safire_b200 import molecule as Mo
from safire_b200.backprop import BackPropagation, mixed_onerdm
from safire_b200.driver import RunParams
from tests import molecule_fixtures as F
from tests.test_molecule_snapshots import CASES, reported_mean

pytestmark = pytest.mark.gpu


def _run(name, with_rdms=False):
    ham, wfn, wt, r = F.snapshot_case(name)
    rp = RunParams(walker_ortho_interval=r["walker_ortho_interval"],
                   population_control_interval=r["population_control_interval"],
                   measure_interval=r["measure_interval"],
                   equilibration_steps=r["equilibration_steps"], seed=r["seed"])
    sim = Mo.simulation(ham, wfn, r["walkers"], r["timestep"], wt, rp, host_fields=True)
    bp = None
    if with_rdms and "bp_steps" in r:
        bp = BackPropagation(sim, wfn.PsiT[0], steps=r["bp_steps"],
                             path_restoration=r["bp_path_restoration"])
    mixed = []
    for step in range(r["steps"]):
        sim.step()
        if with_rdms and "onerdm" in r and step % r["mixed_interval"] == 0:
            g, ws = sim.wfn.OneRDM(sim.wset)
            mixed.append((g / ws).cpu().numpy())
    torch.cuda.synchronize()
    return [v for _, v in sim.energies], mixed, bp, r


@pytest.mark.parametrize("name", CASES)
def test_cuda_path_reproduces_snapshot_energy(cuda, name):
    e, _, _, r = _run(name)
    assert len(e) == r["steps"]
    n = reported_mean(e, r["Energy"][0], tol=1e-8)
    assert n is not None, (np.mean(e), r["Energy"][0])


def _matches_some_length(samples, want, tol=1e-8):
    x = np.asarray(samples)
    for B in range(1, x.shape[0] // 2 + 1):
        n = (x.shape[0] // B) * B
        if np.max(np.abs(x[:n].mean(0) - want)) < tol:
            return True
    return False


@pytest.mark.parametrize("name", ["bh_rhf_closed", "bh_uhf_collinear", "li_rohf_collinear"])
def test_cuda_path_reproduces_snapshot_density_matrices(cuda, name):
    e, mixed, bp, r = _run(name, with_rdms=True)
    want = np.array(r["onerdm"][0]) + 1j * np.array(r["onerdm"][1])
    assert len(mixed) == r["steps"] // r["mixed_interval"]
    assert _matches_some_length(mixed, want)
    want_bp = np.array(r["bp_onerdm"][0]) + 1j * np.array(r["bp_onerdm"][1])
    assert len(bp.samples) == r["steps"] // r["bp_steps"]
    assert _matches_some_length([s[1] for s in bp.samples], want_bp)


@pytest.mark.parametrize("name", ["bh_casci_rhf_phmsd_collinear", "bh_casci_uhf_phmsd_collinear",
                                  "bh_casci_uhf_nomsd_collinear"])
def test_cuda_path_reproduces_snapshot_multireference_backprop(cuda, name):
    """Back propagation over the trial's determinants (44 or 34 references: the PHMSD
    configurations over the rotated complex reference or the orbitals, or the NOMSD
    determinants), each weighted by its share of every walker's overlap; and the mixed
    estimator's density matrix over the same references."""
    from safire_b200 import inputs as I
    from safire_b200.backprop import phmsd_references
    ham, wfn, wt, r = F.snapshot_case(name)
    rp = RunParams(walker_ortho_interval=r["walker_ortho_interval"],
                   population_control_interval=r["population_control_interval"],
                   measure_interval=r["measure_interval"],
                   equilibration_steps=r["equilibration_steps"], seed=r["seed"])
    sim = Mo.simulation(ham, wfn, r["walkers"], r["timestep"], wt, rp, host_fields=True)
    if isinstance(wfn, I.PHMSDInput):
        refs = phmsd_references(I.phmsd_trial(wfn))
    else:
        refs = [(c, P) for c, P in zip(wfn.ci, wfn.PsiT)]
    bp = BackPropagation(sim, steps=r["bp_steps"], path_restoration=r["bp_path_restoration"],
                         references=refs)
    mixed = []
    for step in range(r["steps"]):
        sim.step()
        if step % r["mixed_interval"] == 0:
            mixed.append(mixed_onerdm(sim, refs).cpu().numpy())
    torch.cuda.synchronize()
    assert reported_mean([v for _, v in sim.energies], r["Energy"][0], tol=1e-8) is not None
    want = np.array(r["bp_onerdm"][0]) + 1j * np.array(r["bp_onerdm"][1])
    assert len(bp.samples) == r["steps"] // r["bp_steps"]
    assert _matches_some_length([s[1] for s in bp.samples], want)
    want = np.array(r["onerdm"][0]) + 1j * np.array(r["onerdm"][1])
    assert _matches_some_length(mixed, want)


def test_mixed_onerdm_over_references_equals_the_library_kernel(cuda):
    """For one determinant the reference loop gives the library's afqmc_wfn_onerdm."""
    ham, wfn, wt, r = F.snapshot_case("bh_uhf_collinear")
    rp = RunParams(walker_ortho_interval=10, population_control_interval=1, measure_interval=1,
                   equilibration_steps=0, seed=7)
    sim = Mo.simulation(ham, wfn, 24, 0.01, wt, rp, host_fields=True)
    for _ in range(5):
        sim.step()
    g, ws = sim.wfn.OneRDM(sim.wset)
    got = mixed_onerdm(sim, [(1.0, wfn.PsiT[0])])
    assert torch.max(torch.abs(got - g / ws)).item() < 1e-12
