"""Molecular AFQMC runs from the reference's input files.

`simulation` builds a safire_b200.driver.Simulation from a DenseHamiltonian and a trial read by
safire_b200.inputs: a single NOMSD determinant, several NOMSD determinants (with the
reference's pairwise mean field, NOMSD.cpp:466-520) or a PHMSD expansion (with the reference's
PHMSD mean field, PHMSD.cpp:1330-1572).  `run` drives it with the run_afqmc cadence and returns the
mixed-estimator energies; `blocked_mean` gives their mean and a blocking error bar.

The command line takes the reference's JSON input (the document run_functional.py writes:
`{"seed", "execute": {"walker_set": {"walker_type"}, "wavefunction": {"filename"},
"hamiltonian": {"filename"}, "timestep", "steps", "num_walkers", "population_control_interval",
"measure_interval", "walker_ortho_interval", "equilibration_steps"}}`) and prints the energy:

    python -m safire_b200.molecule afqmc.json
"""
from __future__ import annotations

import json
import math
import sys

import numpy as np
import torch

from . import afqmc as A
from .capi import CLOSED, COLLINEAR
from .driver import RunParams, Simulation
from .inputs import (NOMSDInput, PHMSDInput, molecule_workload, phmsd_trial, read_hamiltonian,
                     read_wavefunction)
from .synth import Workload

WALKER_TYPES = {"CLOSED": CLOSED, "COLLINEAR": COLLINEAR}


def nomsd_mean_field_density(PsiTs, ci, walker_type):
    """The trial density matrix the reference's several-determinant vMF contracts
    (NOMSD.cpp:466-520): over determinant pairs p <= q, the full transition density matrix
    G_qp = A^T (T^-T B^T) with A = PsiT_q, B = PsiT_p^H, T = A B (density_matrix.hpp:535-601),
    weighted by Re(conj(c_q) c_p det T) (one spin factor for CLOSED), summed and divided by the
    sum of the weights.  A pair whose T has an exactly zero LU pivot (orthogonal determinants,
    e.g. occupation patterns in one orbital basis) adds nothing: the reference's getri_or_zero
    returns a zero inverse there and its weight exp(log(0 + DBL_MIN)) underflows to zero.
    Returns [nspin][M][M]."""
    import scipy.linalg as sl
    nspin = 2 if walker_type == COLLINEAR else 1
    M = PsiTs[0][0].shape[1]
    Gsum = np.zeros((nspin, M, M), dtype=np.complex128)
    osum = 0.0
    nd = len(PsiTs)
    for p in range(nd):
        for q in range(p, nd):
            lo = 0j
            Gs = []
            for s in range(nspin):
                Aq = PsiTs[q][s]
                B = PsiTs[p][s].conj().T
                T = Aq @ B
                if T.shape[0] == 0:
                    Gs.append(np.zeros((M, M), dtype=np.complex128))
                    continue
                with np.errstate(all="ignore"):
                    lu, piv = sl.lu_factor(T, check_finite=False)
                d = np.diag(lu)
                if np.any(d == 0):
                    break
                sign = np.prod(np.where(piv != np.arange(piv.size), -1.0, 1.0))
                lo += np.log(sign + 0j) + np.sum(np.log(d.astype(np.complex128)))
                Tinv = sl.lu_solve((lu, piv), np.eye(T.shape[0], dtype=np.complex128))
                Gs.append(Aq.T @ (Tinv.T @ B.T))
            else:
                scl = float((np.conj(ci[q]) * ci[p] * np.exp(lo)).real)
                osum += scl
                for s in range(nspin):
                    Gsum[s] += scl * Gs[s]
    return Gsum / osum


def phmsd_configurations(trial, s):
    """Occupied active orbitals of every unique configuration of spin s, sorted (index 0 the
    reference, then the excitation shells in order)."""
    ref = np.asarray(trial.refc[s])
    out = [np.sort(ref)]
    for n in sorted(trial.exc[s]):
        for e in trial.exc[s][n]:
            c = ref.copy()
            c[e[:n]] = e[n:]
            out.append(np.sort(c))
    return out


def phmsd_mean_field(trial, Likn, dt):
    """PHMSD::vMF (PHMSD.cpp:1330-1572), COLLINEAR, restated on the host: the trial's one-body
    density in the active representation, then the force bias of it.
    - ov_s[u]: det(A_u^H A_u) of each unique configuration's orbitals (A = Orbs[:, conf], Orbs =
      orbmat^H), relative to the reference's (all 1 for orthonormal orbitals);
    - diagonal: each configuration adds w (A^H A)^-T A^T to its rows, w = ov_s[u] sum over its
      determinants of ov_other |coupling|^2;
    - off-diagonal: determinants that share the other spin's configuration and differ by one
      orbital (o1 -> o2) add coupling1 conj(coupling2) orbmat[o1] to row o2 and the conjugate
      weight times orbmat[o2] to row o1, without the overlap factor or the excitation's sign (as
      the reference does; it assumes orthogonal orbitals);
    - divided by sum_k |coupling_k|^2 ov_up ov_dn; then v[n] = sqrt(dt) sum_s sum_{a,m}
      G_s[a][m] Lnak_s[n][a][m] with Lnak built from the active orbitals (Real3Index vbias,
      COLLINEAR).  Returns vMF [Nc] (complex; the propagator keeps its real part)."""
    L = np.asarray(Likn, dtype=np.float64)
    M = trial.M
    orb = [np.asarray(trial.orbmat[s], dtype=np.complex128) for s in (0, 1)]
    Orbs = [o.conj().T for o in orb]
    conf = [phmsd_configurations(trial, s) for s in (0, 1)]
    det = [np.asarray(trial.det_up), np.asarray(trial.det_dn)]
    c2 = np.abs(np.asarray(trial.coef)) ** 2
    coup = np.asarray(trial.coef, dtype=np.complex128)
    ovl = []
    for s in (0, 1):
        lo = []
        for c in conf[s]:
            A = Orbs[s][:, c]
            sign, la = np.linalg.slogdet(A.conj().T @ A)
            lo.append(np.log(sign + 0j) + la)
        lo = np.array(lo)
        o = np.exp(lo - lo[0])
        o[0] = 1.0
        ovl.append(o)
    ov = np.sum(c2 * ovl[0][det[0]] * ovl[1][det[1]])
    G = [np.zeros((orb[s].shape[0], M), dtype=np.complex128) for s in (0, 1)]
    for s in (0, 1):
        o = 1 - s
        for u, c in enumerate(conf[s]):
            ks = np.nonzero(det[s] == u)[0]
            if ks.size == 0:
                continue
            w = ovl[s][u] * np.sum(ovl[o][det[o][ks]] * c2[ks])
            A = Orbs[s][:, c]
            G[s][c] += w * (np.linalg.inv(A.conj().T @ A).T @ A.T)
        for u in range(len(conf[o])):
            ks = np.nonzero(det[o] == u)[0]
            for i1 in range(ks.size):
                c1 = set(conf[s][det[s][ks[i1]]].tolist())
                for i2 in range(i1 + 1, ks.size):
                    c2set = set(conf[s][det[s][ks[i2]]].tolist())
                    d1, d2 = c1 - c2set, c2set - c1
                    if len(d1) != 1:
                        continue
                    o1, o2 = d1.pop(), d2.pop()
                    w = coup[ks[i1]] * np.conj(coup[ks[i2]])
                    G[s][o2] += w * orb[s][o1]
                    G[s][o1] += np.conj(w) * orb[s][o2]
    v = np.zeros(L.shape[3], dtype=np.complex128)
    for s in (0, 1):
        Ls = L[s % L.shape[0]]
        Lnak = np.einsum("ai,imn->amn", orb[s], Ls)
        v += np.einsum("am,amn->n", G[s] / ov, Lnak)
    return math.sqrt(dt) * v


def _workload(ham, wfn, W, dt, walker_type):
    if isinstance(wfn, PHMSDInput):
        trial = phmsd_trial(wfn)
        psi = [np.ascontiguousarray(trial.orbmat[s][trial.refc[s]]) for s in (0, 1)]
        hij = ham.hcore if ham.hcore.shape[0] == 2 else np.concatenate([ham.hcore, ham.hcore])
        E0 = ham.energy_offset(COLLINEAR, wfn.nup, wfn.ndn)
        return Workload("molecule", ham.M, wfn.nup, wfn.ndn, ham.Nc, W, dt, COLLINEAR,
                        np.ascontiguousarray(hij), ham.Likn, E0, psi), trial
    first = NOMSDInput(wfn.walker_type, wfn.M, wfn.nup, wfn.ndn, wfn.ci[:1], wfn.PsiT[:1])
    return molecule_workload(ham, first, W, dt, walker_type), None


def simulation(ham, wfn, W, dt, walker_type=None, rp=None, use_graph=True, host_fields=False):
    """A Simulation of W walkers (FP64) for a trial read by safire_b200.inputs.  The walkers
    start from the determinant with the largest coefficient (NOMSD.cpp:132-153).  A PHMSD run
    starts from the expansion's reference determinant; the reference starts from the
    largest-coefficient configuration (PHMSD.hpp:284-302), the same one when the expansion is
    led by its largest determinant, as the reference's own files are.
    host_fields: draw the fields from the reference's host random stream
    (Simulation.use_host_fields), so that a seeded run reproduces the reference's."""
    rp = rp or RunParams()
    if isinstance(wfn, NOMSDInput) and wfn.ci.size > 1:
        first = int(np.argmax(np.abs(wfn.ci)))
        if first:
            order = [first] + [d for d in range(wfn.ci.size) if d != first]
            wfn = NOMSDInput(wfn.walker_type, wfn.M, wfn.nup, wfn.ndn, wfn.ci[order],
                             [wfn.PsiT[d] for d in order])
    sim = _simulation(ham, wfn, W, dt, walker_type, rp, use_graph)
    if host_fields:
        sim.use_host_fields()
    return sim


def _simulation(ham, wfn, W, dt, walker_type, rp, use_graph):
    wl, trial = _workload(ham, wfn, W, dt, walker_type)
    if trial is not None:
        sim = Simulation.from_workload(wl, W=W, rp=rp, trial=trial,
                                       vMF=phmsd_mean_field(trial, wl.Likn, dt))
        sim.use_graph = False
        return sim
    if wfn.ci.size > 1:
        psis = [[np.ascontiguousarray(p) for p in (d if wl.walker_type == wfn.walker_type
                                                   else [d[0], d[0]])] for d in wfn.PsiT]
        # the pairwise trial density's vbias, through the library's full-G branch
        ham0 = A.HamiltonianOperations(wl.walker_type, wl.M, wl.nup, wl.ndn, wl.Likn, wl.hij,
                                       wl.E0, wl.PsiT)
        hams = [ham0] + [A.HamiltonianOperations(wl.walker_type, wl.M, wl.nup, wl.ndn, wl.Likn,
                                                 wl.hij, wl.E0, P) for P in psis[1:]]
        md = A.NOMSDMulti(hams, wfn.ci)
        G = torch.as_tensor(nomsd_mean_field_density(psis, wfn.ci, wl.walker_type)[None],
                            device="cuda")
        v = torch.empty((1, wl.Nc), dtype=torch.complex128, device="cuda")
        vMF = md.vbias(G.contiguous(), v, dt)[0].cpu().numpy()
        del md, hams, ham0
        sim = Simulation.from_workload(wl, W=W, rp=rp, multidet=(psis, wfn.ci), vMF=vMF)
        # graph-replayed steps are bit-identical to eager ones here and 12% faster at 34
        # determinants (the step is bound by its per-determinant kernels, not by launches)
        sim.use_graph = use_graph
        return sim
    sim = Simulation.from_workload(wl, W=W, rp=rp)
    sim.use_graph = use_graph
    return sim


def run(sim, steps):
    """steps iterations of the run_afqmc loop; returns [(step, energy)] of the measurements."""
    for _ in range(steps):
        sim.step()
    torch.cuda.synchronize()
    return list(sim.energies)


def blocked_mean(x, nblocks=16):
    """Mean of the series x and its error bar from nblocks equal consecutive blocks."""
    x = np.asarray(x, dtype=np.float64)
    nb = max(2, min(nblocks, x.size // 2))
    n = x.size // nb
    blocks = x[x.size - nb * n:].reshape(nb, n).mean(1)
    return float(x.mean()), float(blocks.std(ddof=1) / math.sqrt(nb))


def parse_input(doc):
    """The settings of the reference's JSON input document: {"hamiltonian", "wavefunction" (file
    names), "walkers", "timestep", "steps", "walker_type" (or None: the trial's), "rp"
    (RunParams)}.  The walker count is `num_walkers` (the whole population) or
    `n_walkers_per_mpi_task` (one rank's)."""
    ex = doc["execute"]
    wt = ex.get("walker_set", {}).get("walker_type")
    if wt is not None and wt.upper() not in WALKER_TYPES:
        raise ValueError(f"walker_type {wt} is not supported")
    W = ex.get("num_walkers") or ex.get("n_walkers_per_mpi_task")
    if not W or int(W) <= 0:
        raise ValueError("the input names no walker count")
    rp = RunParams(walker_ortho_interval=int(ex.get("walker_ortho_interval", 5)),
                   population_control_interval=int(ex.get("population_control_interval", 10)),
                   measure_interval=int(ex.get("measure_interval", 10)),
                   equilibration_steps=int(ex.get("equilibration_steps", 100)),
                   seed=int(doc.get("seed", 0)))
    return {"hamiltonian": ex["hamiltonian"]["filename"],
            "wavefunction": ex["wavefunction"]["filename"], "walkers": int(W),
            "timestep": float(ex.get("timestep", 0.01)), "steps": int(ex["steps"]),
            "walker_type": None if wt is None else WALKER_TYPES[wt.upper()], "rp": rp}


def run_input(doc):
    """Run the reference's JSON input document; returns (mean, error, number of measurements)."""
    cfg = parse_input(doc)
    ham = read_hamiltonian(cfg["hamiltonian"])
    wfn = read_wavefunction(cfg["wavefunction"])
    sim = simulation(ham, wfn, cfg["walkers"], cfg["timestep"], cfg["walker_type"], cfg["rp"])
    energies = run(sim, cfg["steps"])
    e = [v for _, v in energies]
    mean, err = blocked_mean(e)
    return mean, err, len(e)


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    if len(argv) != 1:
        print(__doc__)
        return 2
    with open(argv[0]) as fh:
        doc = json.load(fh)
    mean, err, n = run_input(doc)
    print(json.dumps({"energy": mean, "error": err, "measurements": n}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
