"""ORACLE — test infrastructure only (see oracle/__init__.py).

numpy restatement of THCOps, the tensor-hypercontraction HamiltonianOperations
(src/AFQMC/HamiltonianOperations/THCOps.hpp), single determinant, npol = 1, one spin block in
the Hamiltonian (nspin_in_H = 1), no separate rotated factors.  The same interface as
oracle.afqmc.Real3IndexFactorization, so the oracle's NOMSD trial and Propagator run on it.

Factors (THCOps.hpp:50-105): X = Piu [M, nu] (real), Luv [nu, nv] (real), Z = rotMuv [nu, nu]
(real), the trial-rotated points Ydsau [s][a, u] = sum_i PsiT_s[a, i] X[i, u], haj and v0.  They
stand for the Cholesky vectors L_n = X diag(Luv[:, n]) X^T (`cholesky_from_thc`).
"""
from __future__ import annotations

import math

import numpy as np

from .afqmc import CLOSED, COLLINEAR


def cholesky_from_thc(X, Luv):
    """Likn [1, M, M, nv] with L_n[i, k] = sum_u X[i, u] X[k, u] Luv[u, n]."""
    X = np.asarray(X, dtype=np.float64)
    return np.einsum("iu,ku,un->ikn", X, X, np.asarray(Luv, dtype=np.float64))[None]


class THCOps:
    def __init__(self, walker_type, M, nup, ndn, X, Luv, hij, E0, PsiT, Z=None, v0=None):
        self.walker_type = walker_type
        self.M, self.nup, self.ndn = M, nup, ndn
        self.X = np.asarray(X, dtype=np.float64)
        self.Luv = np.asarray(Luv, dtype=np.float64)
        self.nu, self.nCV = self.Luv.shape
        self.Z = self.Luv @ self.Luv.T if Z is None else np.asarray(Z, dtype=np.float64)
        self.hij = np.asarray(hij, dtype=np.complex128)
        self.E0 = float(E0)
        nspin = 2 if walker_type == COLLINEAR else 1
        self.nel = [nup, ndn if walker_type == COLLINEAR else 0]
        ns_h1 = self.hij.shape[0]
        self.haj = np.zeros((self.nel[0] + self.nel[1], M), dtype=np.complex128)
        # Ydsau (rotcXau): the trial's half rotation of the interpolation points
        self.Y = []
        for s in range(nspin):
            if self.nel[s] == 0:
                self.Y.append(np.zeros((0, self.nu), dtype=np.complex128))
                continue
            self.haj[s * nup:s * nup + self.nel[s]] = PsiT[s] @ self.hij[s % ns_h1]
            self.Y.append(np.asarray(PsiT[s], dtype=np.complex128) @ self.X)
        if v0 is None:
            Likn = cholesky_from_thc(self.X, self.Luv)[0]
            v0 = -0.5 * (Likn.reshape(M, -1) @ Likn.reshape(M, -1).T)
        self.vexx = np.asarray(v0, dtype=np.float64).reshape(1, M, M)

    def number_of_cholesky_vectors(self):
        return self.nCV

    def _spin_G(self, G):
        W = G.shape[0]
        nel = self.nel[0] + self.nel[1]
        G3 = G.reshape(W, nel, self.M)
        nspin = 2 if self.walker_type == COLLINEAR else 1
        return [G3[:, s * self.nup:s * self.nup + self.nel[s], :] for s in range(nspin)]

    # Guu_from_compact (THCOps.hpp:636-703): Guu [nu, W]
    def Guu_from_compact(self, G):
        a = 2.0 if self.walker_type == CLOSED else 1.0
        Guu = np.zeros((self.nu, G.shape[0]), dtype=np.complex128)
        for s, Gs in enumerate(self._spin_G(G)):
            if self.nel[s] == 0:
                continue
            Twau = Gs @ self.X  # [W, a, u] = sum_i G[w, a, i] X[i, u]
            Guu += a * np.einsum("wau,au->uw", Twau, self.Y[s])
        return Guu

    # vbias (THCOps.hpp:571-615), ndet == 1: v [W, nv] = sqrt(dt) Luv^T Guu
    def vbias(self, G, dt):
        Guu = self.Guu_from_compact(G)
        return (math.sqrt(dt) * (self.Luv.T @ Guu)).T.copy()

    # vHS (THCOps.hpp:462-569), the complex branch: T[u, w] = sum_v L[u, v] X[w, v];
    # Q[w, i, u] = T[u, w] X[i, u]; v[w] = sqrt(dt) Q[w] X^T.  [1, W, M, M]
    def vHS(self, Xf, dt):
        T = self.Luv @ np.asarray(Xf).T  # [nu, W]
        Q = np.einsum("uw,iu->wiu", T, self.X)
        V = math.sqrt(dt) * np.einsum("wiu,ju->wij", Q, self.X)
        return V[None]

    # Guv_Guu (THCOps.hpp:755-835): Guv [W, nu, nu], diag into Guu [nu, W]
    def _Guv(self, Gs, s):
        Twav = Gs @ self.X  # [W, a, v]
        return np.einsum("au,wav->wuv", self.Y[s], Twav)

    # energy (THCOps.hpp:149-293)
    def energy(self, G, addH1=True, addEJ=True, addEXX=True):
        W = G.shape[0]
        E = np.zeros((W, 3), dtype=np.complex128)
        scl = 2.0 if self.walker_type == CLOSED else 1.0
        spins = self._spin_G(G)
        if addH1:
            E[:, 0] = self.E0
            nel = self.nel[0] + self.nel[1]
            E[:, 0] += scl * np.einsum("wj,j->w", G.reshape(W, nel * self.M),
                                       self.haj.reshape(-1))
        if not (addEJ or addEXX):
            return E
        Guu = np.zeros((self.nu, W), dtype=np.complex128)
        for s, Gs in enumerate(spins):
            if self.nel[s] == 0:
                continue
            Guv = self._Guv(Gs, s)
            Guu += np.einsum("wuu->uw", Guv)
            Guv = Guv * self.Z[None]
            # R[w, u, b] = sum_v Guv[w, u, v] Y[b, v];  T[w, i, b] = sum_u X[i, u] R[w, u, b]
            R = np.einsum("wuv,bv->wub", Guv, self.Y[s])
            T = np.einsum("iu,wub->wib", self.X, R)
            # E[w] += -scl/2 sum_{a, i} T[w, i, a] G[w, a, i]
            E[:, 1] += -0.5 * scl * np.einsum("wia,wai->w", T, Gs)
        if addEJ:
            Tuw = self.Z.T @ Guu
            E[:, 2] += 0.5 * scl * scl * np.einsum("uw,uw->w", Guu, Tuw)
        return E

    # getOneBodyPropagatorMatrix (THCOps.hpp:107-136) + add_one_body_shifts: the same
    # H1 = dt h + dt v0 + vHS(vMF, dt) as the Cholesky form
    def getOneBodyPropagatorMatrix(self, dt, vMF):
        nspin = 2 if self.walker_type == COLLINEAR else 1
        mf = self.vHS(np.asarray(vMF)[None, :], dt)[0, 0]
        H1 = np.zeros((nspin, self.M, self.M), dtype=np.complex128)
        for s in range(nspin):
            H1[s] = dt * self.hij[s % self.hij.shape[0]] + dt * self.vexx[0] + mf
        return H1
