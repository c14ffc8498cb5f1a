"""Molecular AFQMC on the GPU against the reference's statistical references (its functional
tests: BH and N2, 1536 walkers, dt = 0.01, ortho / comb / measurement every 10 steps): the
mixed-estimator energy of each trial agrees with the reference's within four combined standard
errors, and for BH with an RHF trial so does every element of the mixed one-body density
matrix.  Runs are shorter than the reference's (its 12000 or 48000 steps after 3000 of
equilibration), so the allowance comes mostly from this side's error bar."""
import math

import numpy as np
import pytest
import torch

from safire_b200 import molecule as Mo
from safire_b200.driver import RunParams
from tests import molecule_fixtures as F

pytestmark = pytest.mark.gpu


def _run(name, equil, steps, onerdm=False):
    ham, wfn, wt, r = F.case(name)
    rp = RunParams(walker_ortho_interval=r["walker_ortho_interval"],
                   population_control_interval=r["population_control_interval"],
                   measure_interval=r["measure_interval"], equilibration_steps=equil,
                   seed=r["seed"])
    sim = Mo.simulation(ham, wfn, r["walkers"], r["timestep"], wt, rp)
    rdms = []
    for _ in range(equil + steps):
        e = sim.step()
        if onerdm and e is not None:
            rdm, wsum = sim.wfn.OneRDM(sim.wset)
            rdms.append((rdm / wsum).real.cpu().numpy())
    torch.cuda.synchronize()
    energies = [v for _, v in sim.energies]
    return energies, rdms, r


def _check_energy(energies, r):
    m, err = Mo.blocked_mean(energies)
    comb = math.hypot(err, r["energy_error"])
    assert abs(m - r["energy"]) < 4 * comb, (m, err, r["energy"], r["energy_error"])
    return m, err


def test_bh_rhf_closed_energy_and_onerdm(cuda):
    energies, rdms, r = _run("bh_rhf_closed", 3000, 12000, onerdm=True)
    _check_energy(energies, r)
    g = np.array(rdms)[:, 0]                     # [measurements][M][M]
    nb = 16
    n = g.shape[0] // nb
    blocks = g[g.shape[0] - nb * n:].reshape(nb, n, *g.shape[1:]).mean(1)
    mean, err = g.mean(0), blocks.std(0, ddof=1) / math.sqrt(nb)
    ref = np.array(r["onerdm_real"])[0]
    ref_err = np.array(r["onerdm_error_real"])[0]
    assert abs(np.trace(mean) - 3.0) < 1e-10
    # occupied-virtual block (the only fluctuating one in the trial's orbital basis)
    z = np.abs(mean - ref) / np.sqrt(err ** 2 + ref_err ** 2 + 1e-14)
    assert np.max(z) < 5.0, (np.unravel_index(np.argmax(z), z.shape), np.max(z))


def test_bh_uhf_collinear_energy(cuda):
    energies, _, r = _run("bh_uhf_collinear", 3000, 12000)
    _check_energy(energies, r)


def test_bh_casci_nomsd_several_determinants_energy(cuda):
    """34 non-orthogonal-pair NOMSD determinants with the reference's pairwise mean field."""
    energies, _, r = _run("bh_casci_rhf_nomsd_closed", 1000, 5000)
    _check_energy(energies, r)


def test_bh_casci_phmsd_rotated_complex_reference_energy(cuda):
    """PHMSD over a dense complex unitary orbital reference with complex coefficients."""
    energies, _, r = _run("bh_casci_rhf_phmsd_collinear", 1500, 6000)
    _check_energy(energies, r)


def test_n2_cas_phmsd_energy(cuda):
    energies, _, r = _run("n2_cas_phmsd_collinear", 1500, 4500)
    _check_energy(energies, r)
