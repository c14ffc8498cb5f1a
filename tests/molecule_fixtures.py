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
