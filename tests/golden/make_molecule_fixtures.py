"""Extract the molecular inputs and statistical reference energies of the reference's functional
tests into committed fixtures, read with safire_b200's own HDF5 reader.

Writes tests/golden/molecules.npz (Hamiltonians and trial wavefunctions of BH and N2),
tests/golden/molecule_references.json (the statistical references: mixed-estimator energies with
their error bars, the run settings, and the BH RHF mixed-estimator and back-propagated one-body
density matrices) and tests/golden/molecule_snapshots.json (the seeded single-rank snapshots:
energies and density matrices of short runs that a restatement with the same random streams
reproduces to rounding).  Run from the repository
root with the reference checked out at REFERENCE (the argument, else the SAFIRE_REFERENCE
environment variable):

    python tests/golden/make_molecule_fixtures.py [REFERENCE]
"""
import json
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", ".."))

from safire_b200 import inputs as I  # noqa: E402
from safire_b200.h5 import File  # noqa: E402

REF = os.environ.get("SAFIRE_REFERENCE", "")
INP = os.path.join(REF, "tests/functional/afqmc_inputs")
STAT = os.path.join(REF, "tests/functional/statistical_references")
OUT = os.path.dirname(os.path.abspath(__file__))

HAMS = {"bh": "BH/afqmc_H_rhf_closed.h5", "n2": "N2/cas_basis_hamil.h5",
        "bh_spin": "BH/afqmc_H_rhf_collinear.h5", "li": "Li/hamil_closed.h5"}
WFNS = {
    "bh_rhf_nomsd": "BH/afqmc_rhf_nomsd.h5",
    "bh_uhf_nomsd": "BH/afqmc_uhf_nomsd.h5",
    "bh_casci_rhf_nomsd": "BH/afqmc_casci_rhf_nomsd.h5",
    "bh_casci_rhf_phmsd": "BH/afqmc_casci_rhf_phmsd.h5",
    "bh_casci_uhf_phmsd": "BH/afqmc_casci_uhf_phmsd.h5",
    "n2_cas_phmsd": "N2/cas_wfn.h5",
    "bh_casci_rhf_1phmsd": "BH/afqmc_casci_rhf_1phmsd.h5",
    "bh_casci_uhf_1phmsd": "BH/afqmc_casci_uhf_1phmsd.h5",
    "li_rohf_nomsd": "Li/rohf_nomsd_polarized.h5",
    "bh_casci_uhf_nomsd": "BH/afqmc_casci_uhf_nomsd.h5",
}
SNAP = "tests/functional/snapshot_references"
# seeded single-rank snapshots (50 walkers, 20 steps, comb and measurement every step, a 2-step
# back-propagation window where the case has one): (case, hamiltonian, wavefunction, walkers)
SNAPSHOTS = [
    ("bh_rhf_closed", "bh", "bh_rhf_nomsd", "closed", "BH/dense_rhf_basis_closed/rhf_nomsd/closed"),
    ("bh_rhf_collinear", "bh", "bh_rhf_nomsd", "collinear",
     "BH/dense_rhf_basis_closed/rhf_nomsd/collinear"),
    ("bh_uhf_collinear", "bh", "bh_uhf_nomsd", "collinear",
     "BH/dense_rhf_basis_closed/uhf_nomsd/collinear"),
    ("bh_casci_rhf_nomsd_closed", "bh", "bh_casci_rhf_nomsd", "closed",
     "BH/dense_rhf_basis_closed/rcasci_rhf_nomsd/closed"),
    ("bh_casci_rhf_nomsd_collinear", "bh", "bh_casci_rhf_nomsd", "collinear",
     "BH/dense_rhf_basis_closed/rcasci_rhf_nomsd/collinear"),
    ("bh_casci_rhf_phmsd_collinear", "bh", "bh_casci_rhf_phmsd", "collinear",
     "BH/dense_rhf_basis_closed/rcasci_rhf_phmsd/collinear"),
    ("bh_casci_uhf_phmsd_collinear", "bh", "bh_casci_uhf_phmsd", "collinear",
     "BH/dense_rhf_basis_closed/rcasci_uhf_phmsd/collinear"),
    ("bh_casci_rhf_1phmsd_collinear", "bh", "bh_casci_rhf_1phmsd", "collinear",
     "BH/dense_rhf_basis_closed/rcasci_rhf_1phmsd/collinear"),
    ("bh_casci_uhf_1phmsd_collinear", "bh", "bh_casci_uhf_1phmsd", "collinear",
     "BH/dense_rhf_basis_closed/rcasci_uhf_1phmsd/collinear"),
    ("n2_cas_phmsd_collinear", "n2", "n2_cas_phmsd", "collinear",
     "N2/cas_basis_hamil_closed/cas_wfn_collinear/collinear"),
    # the same BH Hamiltonian written with a spin-resolved hcore [2][1][M][1][M]
    ("bh_spinham_rhf_collinear", "bh_spin", "bh_rhf_nomsd", "collinear",
     "BH/dense_rhf_basis_collinear/rhf_nomsd/collinear"),
    ("bh_spinham_uhf_collinear", "bh_spin", "bh_uhf_nomsd", "collinear",
     "BH/dense_rhf_basis_collinear/uhf_nomsd/collinear"),
    ("bh_spinham_casci_rhf_nomsd_collinear", "bh_spin", "bh_casci_rhf_nomsd", "collinear",
     "BH/dense_rhf_basis_collinear/rcasci_rhf_nomsd/collinear"),
    ("bh_spinham_casci_rhf_phmsd_collinear", "bh_spin", "bh_casci_rhf_phmsd", "collinear",
     "BH/dense_rhf_basis_collinear/rcasci_rhf_phmsd/collinear"),
    # Li: a fully polarised ROHF trial, three alpha electrons and an empty beta sector
    ("li_rohf_collinear", "li", "li_rohf_nomsd", "collinear",
     "Li/hamil_closed/rohf_wfn_polarized/collinear"),
    # the UHF-orbital CASCI expansion as COLLINEAR NOMSD determinants
    ("bh_casci_uhf_nomsd_collinear", "bh", "bh_casci_uhf_nomsd", "collinear",
     "BH/dense_rhf_basis_closed/rcasci_uhf_nomsd/collinear"),
]
# (case, hamiltonian, wavefunction, walker type, results.h5 below statistical_references)
CASES = [
    ("bh_rhf_closed", "bh", "bh_rhf_nomsd", "closed", "BH/dense_rhf_basis_closed/rhf_nomsd/closed"),
    ("bh_rhf_collinear", "bh", "bh_rhf_nomsd", "collinear",
     "BH/dense_rhf_basis_closed/rhf_nomsd/collinear"),
    ("bh_uhf_collinear", "bh", "bh_uhf_nomsd", "collinear",
     "BH/dense_rhf_basis_closed/uhf_nomsd/collinear"),
    ("bh_casci_rhf_nomsd_closed", "bh", "bh_casci_rhf_nomsd", "closed",
     "BH/dense_rhf_basis_closed/rcasci_rhf_nomsd/closed"),
    ("bh_casci_rhf_phmsd_collinear", "bh", "bh_casci_rhf_phmsd", "collinear",
     "BH/dense_rhf_basis_closed/rcasci_rhf_phmsd/collinear"),
    ("bh_casci_uhf_phmsd_collinear", "bh", "bh_casci_uhf_phmsd", "collinear",
     "BH/dense_rhf_basis_closed/rcasci_uhf_phmsd/collinear"),
    ("n2_cas_phmsd_collinear", "n2", "n2_cas_phmsd", "collinear",
     "N2/cas_basis_hamil_closed/cas_wfn_collinear/collinear"),
    # the same BH Hamiltonian written with a spin-resolved hcore [2][1][M][1][M]
    ("bh_spinham_rhf_collinear", "bh_spin", "bh_rhf_nomsd", "collinear",
     "BH/dense_rhf_basis_collinear/rhf_nomsd/collinear"),
    ("bh_spinham_uhf_collinear", "bh_spin", "bh_uhf_nomsd", "collinear",
     "BH/dense_rhf_basis_collinear/uhf_nomsd/collinear"),
    ("bh_spinham_casci_rhf_nomsd_collinear", "bh_spin", "bh_casci_rhf_nomsd", "collinear",
     "BH/dense_rhf_basis_collinear/rcasci_rhf_nomsd/collinear"),
    ("bh_spinham_casci_rhf_phmsd_collinear", "bh_spin", "bh_casci_rhf_phmsd", "collinear",
     "BH/dense_rhf_basis_collinear/rcasci_rhf_phmsd/collinear"),
    # Li: a fully polarised ROHF trial, three alpha electrons and an empty beta sector
    ("li_rohf_collinear", "li", "li_rohf_nomsd", "collinear",
     "Li/hamil_closed/rohf_wfn_polarized/collinear"),
]


def _scalar(f, path):
    return complex(np.asarray(f[path]).ravel()[0])


REF_ROOT = [REF]


def main():
    global INP, STAT
    if len(sys.argv) > 1:
        REF_ROOT[0] = sys.argv[1]
        INP = os.path.join(sys.argv[1], "tests/functional/afqmc_inputs")
        STAT = os.path.join(sys.argv[1], "tests/functional/statistical_references")
    if not REF_ROOT[0] or not os.path.isdir(INP):
        sys.exit("give the reference checkout as the argument or in SAFIRE_REFERENCE")
    arrays = {}
    for key, rel in HAMS.items():
        h = I.read_hamiltonian(os.path.join(INP, rel))
        arrays[f"{key}/hcore"] = h.hcore
        arrays[f"{key}/Likn"] = h.Likn
        arrays[f"{key}/energies"] = np.array([h.nuclear_energy, h.frozen_core_energy,
                                              h.madelung_constant])
    for key, rel in WFNS.items():
        w = I.read_wavefunction(os.path.join(INP, rel))
        arrays[f"{key}/meta"] = np.array([w.walker_type, w.M, w.nup, w.ndn])
        arrays[f"{key}/ci"] = w.ci
        if isinstance(w, I.NOMSDInput):
            for d, per_spin in enumerate(w.PsiT):
                for s, p in enumerate(per_spin):
                    arrays[f"{key}/PsiT_{d}_{s}"] = p
        else:
            arrays[f"{key}/occa"] = w.occa
            arrays[f"{key}/occb"] = w.occb
            for r, p in enumerate(w.references):
                arrays[f"{key}/ref_{r}"] = p
    np.savez_compressed(os.path.join(OUT, "molecules.npz"), **arrays)

    refs = {}
    for case, ham, wfn, walker, rel in CASES:
        f = File(os.path.join(STAT, rel, "results.h5"))
        inp = json.loads(str(f["input_file"]))
        ex = inp["execute"]
        m = "measurements/Stage0"
        entry = {
            "hamiltonian": ham, "wavefunction": wfn, "walker_type": walker,
            "energy": _scalar(f, f"{m}/Energy/mean").real,
            "energy_error": _scalar(f, f"{m}/Energy/error").real,
            "components": {k: _scalar(f, f"{m}/{k}/mean").real
                           for k in ("OnebodyEnergy", "CoulombEnergy", "ExchangeEnergy")},
            "walkers": int(np.asarray(f["num_ranks"])) * int(ex.get("n_walkers_per_mpi_task",
                                                                    ex.get("num_walkers", 0))),
            "ranks": int(np.asarray(f["num_ranks"])),
            "steps": ex["steps"], "timestep": ex["timestep"],
            "equilibration_steps": ex["equilibration_steps"],
            "population_control_interval": ex["population_control_interval"],
            "measure_interval": ex["measure_interval"],
            "walker_ortho_interval": ex["walker_ortho_interval"],
            "seed": inp["seed"],
            "run_time_seconds": float(np.asarray(f["run_time_seconds"])),
            "back_propagation": "backprop" in ex.get("estimators", {}),
            "source": f"tests/functional/statistical_references/{rel}/results.h5",
        }
        if case == "bh_rhf_closed":
            g = np.asarray(f[f"{m}/MixedEstimator/OneRDM/mean"])
            ge = np.asarray(f[f"{m}/MixedEstimator/OneRDM/error"])
            entry["onerdm_real"] = g.real.tolist()
            entry["onerdm_error_real"] = ge.real.tolist()
            bp = f"{m}/BackPropEstimator/Steps=100/OneRDM"
            entry["bp_steps"] = 100
            entry["bp_onerdm_real"] = np.asarray(f[f"{bp}/mean"]).real.tolist()
            entry["bp_onerdm_error_real"] = np.asarray(f[f"{bp}/error"]).real.tolist()
            est = inp["execute"]["estimators"]["backprop"]
            entry["bp_path_restoration"] = bool(est.get("path_restoration", True))
        refs[case] = entry
    with open(os.path.join(OUT, "molecule_references.json"), "w") as fh:
        json.dump(refs, fh, indent=1)

    snaps = {}
    for case, ham, wfn, walker, rel in SNAPSHOTS:
        f = File(os.path.join(REF_ROOT[0], SNAP, rel, "results.h5"))
        inp = json.loads(str(f["input_file"]))
        ex = inp["execute"]
        m = "measurements/Stage0"
        est = ex.get("estimators", {})
        entry = {
            "hamiltonian": ham, "wavefunction": wfn, "walker_type": walker,
            "ranks": int(np.asarray(f["num_ranks"])), "walkers": ex["num_walkers"],
            "steps": ex["steps"], "timestep": ex["timestep"], "seed": inp["seed"],
            "equilibration_steps": ex["equilibration_steps"],
            "population_control_interval": ex["population_control_interval"],
            "measure_interval": ex["measure_interval"],
            "walker_ortho_interval": ex["walker_ortho_interval"],
            "source": f"{SNAP}/{rel}/results.h5",
        }
        for k in ("Energy", "OnebodyEnergy", "CoulombEnergy", "ExchangeEnergy"):
            z = _scalar(f, f"{m}/{k}/mean")
            entry[k] = [z.real, z.imag]
        if f"{m}/MixedEstimator/OneRDM/mean" in f:
            g = np.asarray(f[f"{m}/MixedEstimator/OneRDM/mean"])
            entry["mixed_interval"] = est["mixed"]["measure_interval"]
            entry["onerdm"] = [g.real.tolist(), g.imag.tolist()]
        if "backprop" in est:
            n = est["backprop"]["propagation_steps"][0]
            g = np.asarray(f[f"{m}/BackPropEstimator/Steps={n}/OneRDM/mean"])
            entry["bp_steps"] = n
            entry["bp_path_restoration"] = bool(est["backprop"].get("path_restoration", True))
            entry["bp_onerdm"] = [g.real.tolist(), g.imag.tolist()]
        snaps[case] = entry
    with open(os.path.join(OUT, "molecule_snapshots.json"), "w") as fh:
        json.dump(snaps, fh, indent=1)
    print("wrote", len(arrays), "arrays,", len(refs), "references and", len(snaps), "snapshots")


if __name__ == "__main__":
    main()
