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


def make_hamiltonian(M, Nc, decay, seed=0, lscale=0.5):
    """h1 = diag(-2 + 4 i / M) + 0.1 sym(N(0,1)); L_n = lscale decay^n sym(N(0,1)) / sqrt(M)
    (lscale 0.5 in the benchmark construction)."""
    rng = np.random.default_rng(seed)
    h1 = np.diag(-2.0 + 4.0 * np.arange(M) / M) + 0.1 * _sym(rng.standard_normal((M, M)))
    Likn = np.empty((M, M, Nc), dtype=np.float64)
    for n in range(Nc):
        Likn[:, :, n] = lscale * decay ** n * _sym(rng.standard_normal((M, M))) / np.sqrt(M)
    return h1, Likn


def make_workload(name="cfg1", seed=0, W=None, M=None, N=None, Nc=None, lscale=0.5):
    """Build a named workload; W/M/N/Nc override the table (same construction, smaller sizes);
    lscale scales the Cholesky vectors (0.5 in the benchmark construction)."""
    M0, nup, ndn, Nc0, decay, W0, dt = CONFIGS[name]
    M = M or M0
    Nc = Nc or Nc0
    W = W or W0
    if N is not None:
        nup = ndn = N
    h1, Likn = make_hamiltonian(M, Nc, decay, seed, lscale)
    evals, evecs = np.linalg.eigh(h1)
    phi = evecs[:, :nup]
    PsiT = [np.ascontiguousarray(phi.conj().T).astype(np.complex128)]
    return Workload(name, M, nup, ndn, Nc, W, dt, CLOSED,
                    h1[None].astype(np.complex128), Likn[None], 0.0, PsiT)


def make_thc_system(seed=0, M=32, N=8, nu=96, nv=64, W=64, dt=0.01, lscale=0.5,
                    decay=0.97, walker_type=CLOSED):
    """A THC-factorised system (THCOps): h1 as make_hamiltonian, X = Piu [M, nu] the orbitals
    at nu points (N(0,1) / sqrt(M)), Luv [nu, nv] = lscale decay^n N(0,1) / sqrt(nu); the
    Cholesky vectors they stand for are L_n = X diag(Luv[:, n]) X^T (real symmetric).  Returns
    (Workload carrying that Likn, X, Luv); the trial is the N lowest eigenvectors of h1 per spin
    (COLLINEAR: N up, N - 1 down)."""
    rng = np.random.default_rng(seed)
    h1 = np.diag(-2.0 + 4.0 * np.arange(M) / M) + 0.1 * _sym(rng.standard_normal((M, M)))
    X = rng.standard_normal((M, nu)) / np.sqrt(M)
    Luv = np.empty((nu, nv))
    for n in range(nv):
        Luv[:, n] = lscale * decay ** n * rng.standard_normal(nu) / np.sqrt(nu)
    Likn = np.einsum("iu,ku,un->ikn", X, X, Luv)
    _, evecs = np.linalg.eigh(h1)
    nup = N
    ndn = N if walker_type == CLOSED else N - 1
    PsiT = [np.ascontiguousarray(evecs[:, :nup].conj().T).astype(np.complex128)]
    if walker_type == COLLINEAR:
        PsiT.append(np.ascontiguousarray(evecs[:, :ndn].conj().T).astype(np.complex128))
    wl = Workload("thc", M, nup, ndn, nv, W, dt, walker_type, h1[None].astype(np.complex128),
                  Likn[None], 0.0, PsiT)
    return wl, X, Luv


# --------------------------------------------------------------------------------------------
# Particle-hole multi-determinant (PHMSD) trial
# --------------------------------------------------------------------------------------------
@dataclass
class PHMSDTrial:
    """A PHMSD trial in the layout afqmc_phmsd_create takes.

    Per spin s: orbmat[s] [nact_s][M] (the active orbitals, conjugate-transposed), refc[s] [N_s]
    (active orbital of each electron in the reference), exc[s] {nex: [nuniq][2 nex] int32} (the
    unique excitations of that spin, holes as electron indices then particles as active
    orbitals).  Unique index 0 is the reference; then the nex = 1 list, nex = 2, ... in order.
    A determinant k couples unique alpha excitation det_up[k] with unique beta excitation
    det_dn[k] and has coupling coefficient coef[k]: the conjugate of its coefficient c_k in
    |Psi_T> = sum_k c_k |D_k>, as the reference stores the determinant couplings
    (Wavefunction.cpp:458-464), so the overlap is sum_k coef_k <D_k|phi>."""
    M: int
    nup: int
    ndn: int
    orbmat: list
    refc: list
    exc: list
    det_up: np.ndarray
    det_dn: np.ndarray
    coef: np.ndarray

    def unique_count(self, s):
        return 1 + sum(len(v) for v in self.exc[s].values())


def make_phmsd_trial(M, nup, ndn, orbitals, nocc=20, nvirt=40, ndet=4096, max_level=4, seed=0):
    """Reference determinant plus ndet - 1 distinct excitations of levels 1..max_level, each a
    (alpha, beta) pair of excitations confined to the top `nocc` occupied and the lowest `nvirt`
    virtual orbitals of `orbitals` [M][M] (columns = orbitals, lowest first; the same orbitals for
    both spins).  Level L = n_alpha + n_beta is drawn uniformly from 1..max_level and n_alpha
    uniformly from max(0, L - nup_window)..min(L, window); holes and particles are drawn without
    replacement.  Coefficients c = N(0,1) exp(-1.5 L) (the reference's L = 0), normalised."""
    rng = np.random.default_rng(seed)
    nact = max(nup, ndn) + nvirt
    orbmat = np.ascontiguousarray(orbitals[:, :nact].conj().T).astype(np.complex128)
    nel = (nup, ndn)
    uniq = [dict(), dict()]   # spin -> {tuple: index}
    lists = [dict(), dict()]  # spin -> {nex: [tuple]}
    counts = [[1], [1]]

    def key(s, holes, parts):
        n = len(holes)
        if n == 0:
            return 0
        t = tuple(sorted(holes)) + tuple(sorted(parts))
        if t not in uniq[s]:
            uniq[s][t] = None
            lists[s].setdefault(n, []).append(t)
        return t

    # hole windows per spin (a spin with fewer electrons than nocc uses all of them)
    oa, ob = min(nocc, nup), min(nocc, ndn)
    if max_level > min(oa, nvirt) + min(ob, nvirt):
        raise ValueError(f"make_phmsd_trial: level {max_level} needs more than {oa}+{ob} holes "
                         f"or {nvirt} particles per spin")
    dets = {(0, 0)}
    order = [(0, 0)]
    while len(order) < ndet:
        L = int(rng.integers(1, max_level + 1))
        na = int(rng.integers(max(0, L - min(ob, nvirt)), min(L, oa, nvirt) + 1))
        nb = L - na
        ka = key(0, rng.choice(np.arange(nup - oa, nup), na, replace=False).tolist(),
                 rng.choice(np.arange(nup, nup + nvirt), na, replace=False).tolist())
        kb = key(1, rng.choice(np.arange(ndn - ob, ndn), nb, replace=False).tolist(),
                 rng.choice(np.arange(ndn, ndn + nvirt), nb, replace=False).tolist())
        if (ka, kb) in dets:
            continue
        dets.add((ka, kb))
        order.append((ka, kb))
    # unique indices: reference 0, then by excitation number in order of first appearance
    index = [dict(), dict()]
    exc = [dict(), dict()]
    for s in (0, 1):
        k = 1
        for n in sorted(lists[s]):
            exc[s][n] = np.array(lists[s][n], dtype=np.int32).reshape(-1, 2 * n)
            for t in lists[s][n]:
                index[s][t] = k
                k += 1
    det_up = np.array([0 if a == 0 else index[0][a] for a, _ in order], np.int32)
    det_dn = np.array([0 if b == 0 else index[1][b] for _, b in order], np.int32)
    level = np.array([(0 if a == 0 else len(a) // 2) + (0 if b == 0 else len(b) // 2)
                      for a, b in order])
    coef = rng.standard_normal(len(order)) * np.exp(-1.5 * level)
    coef = (coef / np.linalg.norm(coef)).astype(np.complex128)
    refc = [np.arange(nup, dtype=np.int32), np.arange(ndn, dtype=np.int32)]
    return PHMSDTrial(M, nup, ndn, [orbmat, orbmat], refc, exc, det_up, det_dn, coef)


def make_phmsd_workload(seed=0, W=512, M=120, N=30, Nc=960, decay=0.99, dt=0.005, ndet=4096,
                        nocc=20, nvirt=40):
    """The PHMSD benchmark system: COLLINEAR, M=120, N_up=N_dn=30, N_chol=960 (decay 0.99^n), a
    trial of the reference determinant plus ndet - 1 singles-to-quadruples in a 20-occupied /
    40-virtual window (make_phmsd_trial), 512 walkers starting at the reference determinant.
    Returns (Workload, PHMSDTrial)."""
    h1, Likn = make_hamiltonian(M, Nc, decay, seed)
    _, evecs = np.linalg.eigh(h1)
    trial = make_phmsd_trial(M, N, N, evecs, nocc=nocc, nvirt=nvirt, ndet=ndet, seed=seed)
    PsiT = [np.ascontiguousarray(trial.orbmat[s][trial.refc[s]]) for s in (0, 1)]
    wl = Workload("phmsd", M, N, N, Nc, W, dt, COLLINEAR, h1[None].astype(np.complex128),
                  Likn[None], 0.0, PsiT)
    return wl, trial


def phmsd_trial_from_occupations(M, orbmat, refc, occ_up, occ_dn, coef):
    """A PHMSDTrial from a determinant expansion given as occupation lists: orbmat[s] [nact_s][M]
    (active orbitals, conjugate-transposed), refc[s] [N_s] the reference, occ_up / occ_dn
    [ndet][N_s] each determinant's occupied active orbitals in the column order of its coefficient
    coef [ndet] (the wavefunction's c_k).  The particle-hole structure comes from
    afqmc_phmsd_excitations (the library's host code); the permutation signs are folded into the
    coefficients and the result holds their conjugates, the couplings of PHMSDTrial."""
    import ctypes as C

    from . import capi
    occ = [np.ascontiguousarray(occ_up, dtype=np.int32), np.ascontiguousarray(occ_dn, dtype=np.int32)]
    ndet = occ[0].shape[0]
    coef = np.asarray(coef, dtype=np.complex128).copy()
    exc, dets = [dict(), dict()], []
    for s in (0, 1):
        nel = occ[s].shape[1]
        rc = np.ascontiguousarray(refc[s], dtype=np.int32)
        di = np.zeros(ndet, np.int32)
        sg = np.zeros(ndet, np.float64)
        nu = C.c_int()
        nx = np.zeros(max(ndet, 1), np.int32)
        ex = np.zeros(max(ndet * 2 * nel, 1), np.int32)
        ptr = lambda a: a.ctypes.data_as(C.c_void_p)
        capi.call("afqmc_phmsd_excitations", int(orbmat[s].shape[0]), int(nel), ptr(rc),
                  int(ndet), ptr(occ[s]), ptr(di), ptr(sg), C.byref(nu), ptr(nx), ptr(ex))
        coef *= sg
        pos = 0
        for u in range(1, nu.value):
            n = int(nx[u - 1])
            exc[s].setdefault(n, []).append(ex[pos:pos + 2 * n].copy())
            pos += 2 * n
        exc[s] = {n: np.array(v, dtype=np.int32).reshape(-1, 2 * n) for n, v in exc[s].items()}
        dets.append(di)
    return PHMSDTrial(M, occ[0].shape[1], occ[1].shape[1], [np.asarray(o) for o in orbmat],
                      [np.asarray(r, dtype=np.int32) for r in refc], exc, dets[0], dets[1],
                      np.conj(coef))
