"""Seeded synthetic Hamiltonians and trials for the walker-step workloads.

No molecular input ships with this package (the reference reads HDF5 Hamiltonians written by
pyscf, none of which is available here), so every workload is generated from a seed:

  h1   = diag(-2 + 4 i / M) + 0.1 * sym(N(0,1)),   i = orbital index 0..M-1 (real symmetric)
  L_n  = 0.5 * decay**n * sym(N(0,1)) / sqrt(M),   n = 0..Nc-1 (real symmetric)
  E0   = 0
  trial = the N lowest eigenvectors of h1 for each spin (RHF, so CLOSED walkers)

with sym(A) = (A + A^T) / 2 and draws taken in that order from numpy.random.default_rng(seed).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

CLOSED, COLLINEAR = 1, 2


@dataclass
class Workload:
    name: str
    M: int
    nup: int
    ndn: int
    Nc: int
    W: int
    dt: float
    walker_type: int
    hij: np.ndarray      # complex [1, M, M]
    Likn: np.ndarray     # float64 [1, M, M, Nc]
    E0: float
    PsiT: list           # complex [N_s, M] per spin (one entry for CLOSED)


CONFIGS = {
    # name: (M, N_up, N_dn, Nc, decay, W, dt)
    "cfg1": (32, 8, 8, 128, 0.97, 64, 0.01),
    "cfg2": (200, 50, 50, 1600, 0.995, 1024, 0.005),
}


def _sym(a):
    return 0.5 * (a + a.T)


def make_hamiltonian(M, Nc, decay, seed=0):
    rng = np.random.default_rng(seed)
    h1 = np.diag(-2.0 + 4.0 * np.arange(M) / M) + 0.1 * _sym(rng.standard_normal((M, M)))
    Likn = np.empty((M, M, Nc), dtype=np.float64)
    for n in range(Nc):
        Likn[:, :, n] = 0.5 * decay ** n * _sym(rng.standard_normal((M, M))) / np.sqrt(M)
    return h1, Likn


def make_workload(name="cfg1", seed=0, W=None, M=None, N=None, Nc=None):
    """Build a named workload; W/M/N/Nc override the table (same construction, smaller sizes)."""
    M0, nup, ndn, Nc0, decay, W0, dt = CONFIGS[name]
    M = M or M0
    Nc = Nc or Nc0
    W = W or W0
    if N is not None:
        nup = ndn = N
    h1, Likn = make_hamiltonian(M, Nc, decay, seed)
    evals, evecs = np.linalg.eigh(h1)
    phi = evecs[:, :nup]
    PsiT = [np.ascontiguousarray(phi.conj().T).astype(np.complex128)]
    return Workload(name, M, nup, ndn, Nc, W, dt, CLOSED,
                    h1[None].astype(np.complex128), Likn[None], 0.0, PsiT)
