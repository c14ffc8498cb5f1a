"""Loaders for the molecular fixtures in tests/golden (written by
tests/golden/make_molecule_fixtures.py from the reference's functional-test inputs)."""
import json
import os

import numpy as np

from safire_b200 import inputs as I

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
_npz = None


def _data():
    global _npz
    if _npz is None:
        _npz = np.load(os.path.join(GOLDEN, "molecules.npz"))
    return _npz


def references():
    with open(os.path.join(GOLDEN, "molecule_references.json")) as fh:
        return json.load(fh)


def hamiltonian(key):
    d = _data()
    nuc, fzc, mad = (float(x) for x in d[f"{key}/energies"])
    return I.DenseHamiltonian(d[f"{key}/hcore"], d[f"{key}/Likn"], nuc, fzc, mad)


def wavefunction(key):
    d = _data()
    wt, M, nup, ndn = (int(x) for x in d[f"{key}/meta"])
    ci = d[f"{key}/ci"]
    if f"{key}/occa" in d:
        refs = []
        while f"{key}/ref_{len(refs)}" in d:
            refs.append(d[f"{key}/ref_{len(refs)}"])
        return I.PHMSDInput(wt, M, nup, ndn, ci, d[f"{key}/occa"], d[f"{key}/occb"], refs)
    nspin = 2 if wt == I.COLLINEAR else 1
    psi = [[d[f"{key}/PsiT_{k}_{s}"] for s in range(nspin)] for k in range(ci.size)]
    return I.NOMSDInput(wt, M, nup, ndn, ci, psi)


def case(name):
    """(DenseHamiltonian, wavefunction input, walker type, reference entry) of a case."""
    r = references()[name]
    wt = {"closed": I.CLOSED, "collinear": I.COLLINEAR}[r["walker_type"]]
    return hamiltonian(r["hamiltonian"]), wavefunction(r["wavefunction"]), wt, r


def snapshots():
    with open(os.path.join(GOLDEN, "molecule_snapshots.json")) as fh:
        return json.load(fh)


def snapshot_case(name):
    """(DenseHamiltonian, wavefunction input, walker type, snapshot entry)."""
    r = snapshots()[name]
    wt = {"closed": I.CLOSED, "collinear": I.COLLINEAR}[r["walker_type"]]
    return hamiltonian(r["hamiltonian"]), wavefunction(r["wavefunction"]), wt, r


def oracle_snapshot_run(name):
    """The oracle's run_afqmc on a snapshot case with the reference's host random streams:
    returns the per-step mixed-estimator energies."""
    from oracle import afqmc as O
    from oracle import phmsd as OP
    from safire_b200 import molecule as Mo
    ham, wfn, wt, r = snapshot_case(name)
    dt = r["timestep"]
    wl, trial = Mo._workload(ham, wfn if not (isinstance(wfn, I.NOMSDInput) and wfn.ci.size > 1)
                             else I.NOMSDInput(wfn.walker_type, wfn.M, wfn.nup, wfn.ndn,
                                               wfn.ci[:1], wfn.PsiT[:1]), r["walkers"], dt, wt)
    if trial is not None:
        oham = O.Real3IndexFactorization(I.COLLINEAR, wl.M, wl.nup, wl.ndn, wl.Likn, wl.hij,
                                         wl.E0, wl.PsiT)
        owfn = OP.PHMSDWavefunction(trial, oham, wl.Likn, wl.hij,
                                    Mo.phmsd_mean_field(trial, wl.Likn, dt))
    elif wfn.ci.size > 1:
        psis = [d if wl.walker_type == wfn.walker_type else [d[0], d[0]] for d in wfn.PsiT]
        ohams = [O.Real3IndexFactorization(wl.walker_type, wl.M, wl.nup, wl.ndn, wl.Likn, wl.hij,
                                           wl.E0, P) for P in psis]
        G = Mo.nomsd_mean_field_density(psis, wfn.ci, wl.walker_type)
        owfn = O.NOMSDMulti(ohams, psis, wfn.ci, O.full_g_vbias(wl.Likn, G, dt, wl.walker_type))
    else:
        oham = O.Real3IndexFactorization(wl.walker_type, wl.M, wl.nup, wl.ndn, wl.Likn, wl.hij,
                                         wl.E0, wl.PsiT)
        owfn = O.NOMSD(oham, wl.PsiT)
    prop = O.Propagator(owfn, O.PropagatorParams(dt=dt))
    ws = O.WalkerSet.from_trial(owfn, r["walkers"])
    rp = O.RunParams(steps=r["steps"], walker_ortho_interval=r["walker_ortho_interval"],
                     population_control_interval=r["population_control_interval"],
                     measure_interval=r["measure_interval"],
                     equilibration_steps=r["equilibration_steps"], seed=r["seed"])
    en, _ = O.run_afqmc(owfn, prop, ws, rp)
    return [e for _, e in en], r
