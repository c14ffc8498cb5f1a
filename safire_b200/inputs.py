"""Hamiltonian and trial-wavefunction input files in the reference's HDF5 format.

- Hamiltonian (RealDenseHamiltonian.cpp:74-134): group `Hamiltonian` with `hcore`
  [nspin][npol][M][npol][M] (real, or complex as a trailing {re, im} axis or compound),
  `DenseFactorized/L` [nspin_H2][1][M][1][M][Nc] (real) and the energy offset
  E0 = nuclear_energy + frozen_core_energy - nelec * madelung_constant from the group's attributes
  (hdf5_helpers.hpp:84-106).
- Wavefunction (readWfn.cpp:66-115, readWfn.h:88-150): group `Wavefunction/NOMSD` or
  `Wavefunction/PHMSD` with the `spin_type` attribute ("closed" / "collinear" / "noncollinear"),
  `ci_coeffs`, and either sparse matrices `PsiT_k` (NOMSD: determinant d, spin s at
  k = d * nspin + s) or occupation lists `occa` / `occb` [ndet][N_s] over the rows of the optional
  orbital references `PsiT_0` (, `PsiT_1`) (PHMSD, readWfn.cpp:150-215).
- Sparse matrix (csr_utils.hpp:344-420): `shape` (nrows, ncols), `row_pointers`,
  `column_indices`, `values`; or the legacy `dims` (nrows, ncols, nnz), `pointers_begin_`,
  `pointers_end_`, `jdata_`, `data_`.

The readers return host numpy arrays in the layouts HamiltonianOperations, NOMSD and PHMSD take
(safire_b200.afqmc); `molecule_workload` assembles a single-determinant run and
`phmsd_trial` a particle-hole trial.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .capi import CLOSED, COLLINEAR
from .h5 import File

NONCOLLINEAR = 3  # the reference's walker-type enum value; read, never run

SPIN_TYPES = {"closed": CLOSED, "collinear": COLLINEAR, "noncollinear": NONCOLLINEAR}


def _complex(a, ndim):
    """A complex array of rank ndim from a real one, a complex one, or a real one with a trailing
    {re, im} axis (rank ndim + 1)."""
    a = np.asarray(a)
    if a.ndim == ndim + 1 and a.shape[-1] == 2 and a.dtype.kind == "f":
        return a[..., 0] + 1j * a[..., 1]
    return a.astype(np.complex128)


def read_csr(f, path):
    """Dense complex matrix of the sparse matrix stored in group `path`."""
    if f"{path}/shape" in f:
        nrows, ncols = (int(x) for x in f[f"{path}/shape"])
        ptr = np.asarray(f[f"{path}/row_pointers"], dtype=np.int64)
        if ptr.shape != (nrows + 1,) or ptr[0] != 0:
            raise ValueError(f"{path}: bad row_pointers")
        begin, end = ptr[:-1], ptr[1:]
        cols = np.asarray(f[f"{path}/column_indices"], dtype=np.int64)
        vals = _complex(f[f"{path}/values"], 1)
    else:  # legacy layout
        dims = [int(x) for x in f[f"{path}/dims"]]
        nrows, ncols = dims[0], dims[1]
        begin = np.asarray(f[f"{path}/pointers_begin_"], dtype=np.int64)
        end = np.asarray(f[f"{path}/pointers_end_"], dtype=np.int64)
        cols = np.asarray(f[f"{path}/jdata_"], dtype=np.int64)
        vals = _complex(f[f"{path}/data_"], 1)
    out = np.zeros((nrows, ncols), dtype=np.complex128)
    for r in range(nrows):
        out[r, cols[begin[r]:end[r]]] += vals[begin[r]:end[r]]
    return out


@dataclass
class DenseHamiltonian:
    hcore: np.ndarray  # complex [nspin_H1][M][M]
    Likn: np.ndarray   # float64 [nspin_H2][M][M][Nc]
    nuclear_energy: float
    frozen_core_energy: float
    madelung_constant: float

    @property
    def M(self):
        return self.hcore.shape[-1]

    @property
    def Nc(self):
        return self.Likn.shape[-1]

    def energy_offset(self, walker_type, nup, ndn):
        """hdf5_helpers.hpp:84-106: nuclear + frozen core - nelec * madelung."""
        nelec = 2 * nup if walker_type == CLOSED else nup + ndn
        return self.nuclear_energy + self.frozen_core_energy - nelec * self.madelung_constant


def read_hamiltonian(path):
    f = File(path)
    at = f.attrs("Hamiltonian")
    h = np.asarray(f["Hamiltonian/hcore"])
    if h.dtype.kind == "f" and h.ndim == 6 and h.shape[-1] == 2:
        h = h[..., 0] + 1j * h[..., 1]
    if h.ndim != 5 or h.shape[1] != 1 or h.shape[3] != 1:
        raise ValueError(f"hcore has shape {h.shape}; expected [nspin][1][M][1][M] (spinor "
                         "Hamiltonians are not supported)")
    ns, _, M, _, _ = h.shape
    hcore = h.reshape(ns, M, M).astype(np.complex128)
    L = np.asarray(f["Hamiltonian/DenseFactorized/L"])
    if L.dtype.kind == "c" or (L.ndim == 7 and L.shape[-1] == 2):
        raise ValueError("complex Cholesky vectors are not supported (the factorisation is real)")
    if L.ndim != 6 or L.shape[1] != 1 or L.shape[3] != 1 or L.shape[2] != M or L.shape[4] != M:
        raise ValueError(f"DenseFactorized/L has shape {L.shape}; expected [nspin][1][M][1][M][Nc]")
    if L.shape[0] not in (1, ns):
        raise ValueError(f"DenseFactorized/L has nspin {L.shape[0]}, expected 1 or {ns}")
    Likn = np.ascontiguousarray(L.reshape(L.shape[0], M, M, L.shape[5]), dtype=np.float64)
    return DenseHamiltonian(hcore, Likn, float(at.get("nuclear_energy", 0.0)),
                            float(at.get("frozen_core_energy", 0.0)),
                            float(at.get("madelung_constant", 0.0)))


@dataclass
class NOMSDInput:
    walker_type: int
    M: int
    nup: int
    ndn: int
    ci: np.ndarray       # complex [ndet]
    PsiT: list           # PsiT[d][s] complex [N_s][M]


@dataclass
class PHMSDInput:
    walker_type: int
    M: int
    nup: int
    ndn: int
    ci: np.ndarray       # complex [ndet], first coefficient made real-positive
    occa: np.ndarray     # int [ndet][nup], rows of the alpha reference (or orbitals)
    occb: np.ndarray     # int [ndet][ndn], unshifted
    references: list     # [] or the dense PsiT_0 (, PsiT_1) [nact][M]


def read_wavefunction(path):
    """NOMSDInput or PHMSDInput of the first wavefunction group in the file (NOMSD first, as
    readWfn.cpp:50-62 with type "any")."""
    f = File(path)
    kind = "NOMSD" if "Wavefunction/NOMSD" in f else "PHMSD"
    g = f"Wavefunction/{kind}"
    at = f.attrs(g)
    if "spin_type" in at:
        wt = SPIN_TYPES[str(at["spin_type"]).lower()]
    elif f"{g}/dims" in f:
        wt = int(f[f"{g}/dims"][3])
    else:
        raise ValueError(f"{path}: no spin_type attribute")
    ci = _complex(f[f"{g}/ci_coeffs"], 1).reshape(-1)
    if kind == "PHMSD":
        occa = np.asarray(f[f"{g}/occa"], dtype=np.int64)
        occb = np.asarray(f[f"{g}/occb"], dtype=np.int64)
        refs = []
        while f"{g}/PsiT_{len(refs)}" in f:
            refs.append(read_csr(f, f"{g}/PsiT_{len(refs)}"))
        M = int(at["number_of_orbitals"])
        ci = ci * (-1.0 if ci[0].real < 0 else 1.0)  # readWfn.cpp:162-163
        return PHMSDInput(wt, M, occa.shape[1], occb.shape[1], ci, occa, occb, refs)
    nspin = 2 if wt == COLLINEAR else 1
    psi = []
    for d in range(ci.size):
        psi.append([read_csr(f, f"{g}/PsiT_{d * nspin + s}") for s in range(nspin)])
    nup = psi[0][0].shape[0]
    ndn = psi[0][1].shape[0] if wt == COLLINEAR else (nup if wt == CLOSED else 0)
    npol = 2 if wt == NONCOLLINEAR else 1
    return NOMSDInput(wt, psi[0][0].shape[1] // npol, nup, ndn, ci, psi)


def molecule_workload(ham, wfn, W, dt, walker_type=None, name="molecule"):
    """A safire_b200.synth.Workload for a single-determinant NOMSD trial; walker_type defaults to
    the wavefunction's (a CLOSED trial runs COLLINEAR walkers when asked, readWfn.h:123-133)."""
    from .synth import Workload
    if not isinstance(wfn, NOMSDInput):
        raise TypeError("molecule_workload takes a NOMSD wavefunction")
    if wfn.ci.size != 1:
        raise ValueError("molecule_workload builds single-determinant runs")
    wt = wfn.walker_type if walker_type is None else walker_type
    if wt == NONCOLLINEAR:
        raise ValueError("NONCOLLINEAR walkers are not supported")
    psi = wfn.PsiT[0]
    if wt == COLLINEAR and wfn.walker_type == CLOSED:
        psi = [psi[0], psi[0]]
    elif wt != wfn.walker_type:
        raise ValueError("the trial's spin type cannot be converted to these walkers")
    if ham.M != wfn.M:
        raise ValueError(f"Hamiltonian has {ham.M} orbitals, the wavefunction {wfn.M}")
    hij = ham.hcore
    if wt == COLLINEAR and hij.shape[0] == 1:
        hij = np.concatenate([hij, hij])
    nup = psi[0].shape[0]
    ndn = psi[1].shape[0] if wt == COLLINEAR else nup
    E0 = ham.energy_offset(wt, nup, ndn)
    return Workload(name, ham.M, nup, ndn, ham.Nc, W, dt, wt, np.ascontiguousarray(hij),
                    ham.Likn, E0, [np.ascontiguousarray(p) for p in psi])


def phmsd_trial(wfn):
    """safire_b200.synth.PHMSDTrial of a PHMSD wavefunction (COLLINEAR): the active orbitals are
    the rows of the orbital references (PsiT_0 for alpha, the last one for beta) or the identity,
    the reference determinant is the first row of occa / occb, and the permutation signs of the
    excitations are folded into the coefficients."""
    from .synth import phmsd_trial_from_occupations
    if not isinstance(wfn, PHMSDInput):
        raise TypeError("phmsd_trial takes a PHMSD wavefunction")
    if wfn.walker_type != COLLINEAR:
        raise ValueError("PHMSD trials need COLLINEAR walkers")
    if wfn.references:
        orb = [wfn.references[0], wfn.references[-1]]
    else:
        orb = [np.eye(wfn.M, dtype=np.complex128)] * 2
    refc = [wfn.occa[0], wfn.occb[0]]
    return phmsd_trial_from_occupations(wfn.M, [np.ascontiguousarray(o) for o in orb], refc,
                                        wfn.occa, wfn.occb, wfn.ci)
