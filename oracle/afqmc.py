"""ORACLE — test infrastructure only (see oracle/__init__.py).

numpy / scipy restatement of the reference's CPU path for the batched phaseless AFQMC walker step.
The dense linear algebra goes through the same LAPACK routines the reference's CPU build reaches
through TRIQS nda (zgetrf, zgetri, zgeqrf, zungqr, zheev); everything SAFIRE computes itself
(log-determinant conventions, Taylor propagation, force-bias fields, phaseless update, comb) is
restated line by line.  Every function names the reference lines it follows; paths are relative
to the reference repository root.

Conventions: complex128 everywhere; arrays are C-ordered like the reference's nda views.
  S   [W, M, N]   walker Slater matrices (one spin block)
  A   [N, M]      PsiT (the trial's conjugate transpose, "herm" form)
  G   [W, N, M]   half-rotated mixed density matrix (compact form)
"""
from __future__ import annotations

import ctypes
import math
import os
from dataclasses import dataclass, field

import numpy as np
import scipy.linalg.lapack as lapack

DBL_MIN = np.finfo(np.float64).tiny
PI = math.pi

CLOSED, COLLINEAR = 1, 2  # reference enum WALKER_TYPES (src/AFQMC/config.h:46-52)

# walker_data properties, in walker-row order (src/AFQMC/Walkers/WalkerSetBase.cpp:88-110)
WEIGHT, PHASE, PSEUDO_ELOC, E1, EXX, EJ, OVLP, LOGSCL_UP, LOGSCL_DN, IS_UNITARY, THETA = range(11)
NPROP = 11


# --------------------------------------------------------------------------------------------
# RNG (C part: oracle/rng.c)
# --------------------------------------------------------------------------------------------
_LIB = None


def _lib():
    global _LIB
    if _LIB is None:
        here = os.path.dirname(os.path.abspath(__file__))
        path = os.path.join(here, "_build", "liboracle.so")
        if not os.path.exists(path):
            import subprocess
            subprocess.check_call(["make", "-s", "-C", here, "all"])
        lib = ctypes.CDLL(path)
        lib.oracle_split_seed.restype = ctypes.c_uint64
        lib.oracle_split_seed.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_uint]
        lib.oracle_mt_state_size.restype = ctypes.c_int
        lib.oracle_mt_seed.argtypes = [ctypes.c_void_p, ctypes.c_uint32]
        lib.oracle_mt_canonical.restype = ctypes.c_double
        lib.oracle_mt_canonical.argtypes = [ctypes.c_void_p]
        lib.oracle_mt_fill_uniform.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_long]
        lib.oracle_comb.restype = ctypes.c_int
        lib.oracle_comb.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_void_p]
        _LIB = lib
    return _LIB


def split_seed(seed: int, rank: int, stream: int) -> int:
    """splitmix64 seed split (src/utilities/Random.cpp:7-20)."""
    return int(_lib().oracle_split_seed(seed, rank, stream))


class HostRandomGenerator:
    """std::mt19937 + uniform_real_distribution<double>(0,1) (src/utilities/Random.hpp:37-51)."""

    def __init__(self, seed64: int):
        lib = _lib()
        self._state = ctypes.create_string_buffer(lib.oracle_mt_state_size())
        lib.oracle_mt_seed(self._state, ctypes.c_uint32(seed64 & 0xFFFFFFFF))

    def sample_uniform(self, n: int) -> np.ndarray:
        out = np.empty(n, dtype=np.float64)
        _lib().oracle_mt_fill_uniform(self._state, out.ctypes.data, n)
        return out


def comb(rng: HostRandomGenerator, weights: np.ndarray, num_target: int) -> np.ndarray:
    """Comb branching (src/AFQMC/Walkers/population_control.hpp:34-65)."""
    w = np.ascontiguousarray(weights, dtype=np.float64)
    off = np.zeros(w.size, dtype=np.int32)
    rc = _lib().oracle_comb(rng._state, w.ctypes.data, w.size, num_target, off.ctypes.data)
    if rc != 0:
        raise RuntimeError("The total walker weight collapsed")
    return off


def plan_walker_exchange(offspring, counts):
    """Deterministic cross-rank exchange plan (population_control.hpp:87-133).

    Returns a list of (src, walker, dst, copies)."""
    offspring = np.asarray(offspring)
    ntot = int(sum(counts))
    if offspring.size != ntot:
        raise ValueError("plan_walker_exchange: size mismatch")
    if int(offspring.sum()) != ntot:
        raise ValueError("plan_walker_exchange: offspring does not preserve the population")
    exports, deficits = [], []
    first = 0
    for r, nw in enumerate(counts):
        local = offspring[first:first + nw]
        excess = int(local.sum()) - nw
        if excess < 0:
            deficits.append([r, -excess])
        if excess > 0:
            order = sorted(range(nw), key=lambda a: -int(local[a]))  # stable sort, descending
            k = 0
            while excess > 0:
                m = min(int(local[order[k]]), excess)
                exports.append([r, order[k], m])
                excess -= m
                k += 1
        first += nw
    plan = []
    d = 0
    for src, wk, copies in exports:
        while copies > 0:
            n = min(copies, deficits[d][1])
            plan.append((src, wk, deficits[d][0], n))
            copies -= n
            deficits[d][1] -= n
            if deficits[d][1] == 0:
                d += 1
    return plan


def single_rank_slot_map(offspring: np.ndarray) -> np.ndarray:
    """Source walker of every slot after swap_walkers_async on one rank
    (population_control.hpp:142-209 with an empty plan): a walker with keep>=1 stays in its slot,
    its extra copies fill the slots of the walkers with keep==0 in increasing order."""
    off = np.asarray(offspring)
    nw = off.size
    src = np.arange(nw)
    free = [i for i in range(nw) if off[i] == 0]
    nxt = 0
    for i in range(nw):
        for _ in range(1, int(off[i])):
            src[free[nxt]] = i
            nxt += 1
    assert nxt == len(free)
    return src


def swap_walkers_slot_map(offspring, counts, me):
    """Global source walker of every slot of rank `me` after swap_walkers_async
    (population_control.hpp:142-209): local keepers stay, arrivals take the freed slots in plan
    order, then the extra local copies (walker order) and the extra copies of each arrival fill
    the remaining freed slots.  Global index = counts[0] + ... + counts[r-1] + local index."""
    offspring = np.asarray(offspring)
    counts = [int(c) for c in counts]
    plan = plan_walker_exchange(offspring, counts)
    first = int(sum(counts[:me]))
    nw = counts[me]
    keep = [int(x) for x in offspring[first:first + nw]]
    for src, wk, dst, copies in plan:
        if src == me:
            keep[wk] -= copies
    src_of = list(range(first, first + nw))
    free = [i for i in range(nw) if keep[i] == 0]
    nxt = 0
    arrivals = []
    for src, wk, dst, copies in plan:
        if src != me and dst == me:
            slot = free[nxt]
            nxt += 1
            src_of[slot] = int(sum(counts[:src])) + wk
            arrivals.append((slot, copies))
    for i in range(nw):
        for _ in range(1, keep[i]):
            src_of[free[nxt]] = first + i
            nxt += 1
    for slot, copies in arrivals:
        for _ in range(1, copies):
            src_of[free[nxt]] = src_of[slot]
            nxt += 1
    if nxt != len(free):
        raise ValueError("swap_walkers_slot_map: %d slots left unfilled" % (len(free) - nxt))
    return np.asarray(src_of)


# --------------------------------------------------------------------------------------------
# Determinants (src/numerics/operations/determinants_impl.hpp)
# --------------------------------------------------------------------------------------------
def _wrap_imag(z: complex) -> complex:
    im = z.imag
    if im > PI:
        while im > PI:
            im -= 2 * PI
    elif im < -PI:
        while im < -PI:
            im += 2 * PI
    return complex(z.real, im)


def log_det_from_getrf(lu: np.ndarray, piv: np.ndarray, res: complex) -> complex:
    """res += sum_i log(+-U_ii + DBL_MIN), sign flipped where the 1-based pivot != i+1; then the
    imaginary part of the accumulated value is brought to [-pi, pi]
    (determinants_impl.hpp:32-75)."""
    n = lu.shape[0]
    for i in range(n):
        d = complex(lu[i, i])
        if piv[i] == i + 1:
            res += np.log(d + DBL_MIN)
        else:
            res += np.log(complex(-1.0, 0.0) * d + DBL_MIN)
    return _wrap_imag(complex(res))


def log_det_from_geqrf(r: np.ndarray, res: complex):
    """scl_i = -1 if Re R_ii < 0 else 1; res += sum log(scl_i R_ii + DBL_MIN), no wrap
    (determinants_impl.hpp:77-108).  Returns (res, scl)."""
    n = min(r.shape)
    scl = np.ones(n, dtype=np.complex128)
    for i in range(n):
        if r[i, i].real < 0:
            scl[i] = -1.0
        res += np.log(scl[i] * r[i, i] + DBL_MIN)
    return complex(res), scl


def _getrf_ref(T: np.ndarray):
    """LAPACK getrf as nda calls it on a C-ordered matrix: LAPACK sees T^T (column-major)."""
    lu, piv, info = lapack.zgetrf(np.ascontiguousarray(T.T))
    return lu, piv + 1, info  # scipy returns 0-based pivots


def _getri_or_zero_ref(lu, piv1):
    """getri_or_zero (src/numerics/nda_functions.hpp:422-439): inverse, or zero if singular.
    lu/piv1 are the factors of T^T, so the inverse of T^T comes back; transposed -> T^{-1}."""
    inv, info = lapack.zgetri(lu, piv1 - 1)
    if info != 0:
        return np.zeros_like(lu)
    return np.ascontiguousarray(inv.T)


# --------------------------------------------------------------------------------------------
# det_ops (src/AFQMC/SlaterDeterminantOperations/density_matrix.hpp)
# --------------------------------------------------------------------------------------------
def log_overlap_impl(A, B, ovlp, herm=True, invert=False):
    """T = A*B (herm) or A^H*B, LU, ovlp += log det, optional inverse
    (density_matrix.hpp:113-156).  Returns TNN [W,N,N] (the inverse when invert)."""
    W, NMO, NEL = B.shape
    TNN = np.zeros((W, NEL, NEL), dtype=np.complex128)
    if NEL == 0:
        return TNN
    for w in range(W):
        T = A @ B[w] if herm else A.conj().T @ B[w]
        lu, piv1, info = _getrf_ref(T)
        ovlp[w] = log_det_from_getrf(lu, piv1, complex(ovlp[w]))
        TNN[w] = _getri_or_zero_ref(lu, piv1) if invert else lu.T
    return TNN


def Log_Overlap(A, B, ovlp):
    """(density_matrix.hpp:431-447)"""
    log_overlap_impl(A, B, ovlp, herm=True, invert=False)


def MixedDensityMatrix(A, B, ovlp, compact=True, herm=True):
    """(density_matrix.hpp:535-601).  compact: G = T^{-T} B^T  [W,N,M];
    full (herm): G = A^T (T^{-T} B^T)  [W,M,M]."""
    W, NMO, NEL = B.shape
    if NEL == 0:
        return np.zeros((W, NEL, NMO) if compact else (W, NMO, NMO), dtype=np.complex128)
    TNN = log_overlap_impl(A, B, ovlp, herm, True)
    C = np.matmul(np.swapaxes(TNN, 1, 2), np.swapaxes(B, 1, 2))  # product<'T','T'>(TNN,B,C)
    if compact:
        return C
    if herm:
        return np.matmul(A.T, C)  # product<'T'>(A,TNM,C)
    raise NotImplementedError


def inverse_logdet(A, ovlp):
    """Batched inverse and log det (density_matrix.hpp:80-111).  Returns the inverses."""
    W, N, _ = A.shape
    out = np.zeros_like(A)
    for w in range(W):
        lu, piv1, info = _getrf_ref(A[w])
        ovlp[w] = log_det_from_getrf(lu, piv1, complex(ovlp[w]))
        out[w] = _getri_or_zero_ref(lu, piv1)
    return out


def orthogonalize(S, log_detR):
    """In-place QR re-orthonormalisation of S [W,M,N] (orthogonalize.hpp:131-169):
    geqrf + ungqr on S (M x N, column-major view of the transposed copy), log det R with the
    sign fix, S <- Q * diag(scl)."""
    W, M, N = S.shape
    if S.size == 0:
        return
    for w in range(W):
        qr, tau, work, info = lapack.zgeqrf(np.asfortranarray(S[w]))
        res, scl = log_det_from_geqrf(qr[:N, :N], complex(log_detR[w]))
        log_detR[w] = res
        q, work, info = lapack.zungqr(qr[:, :N], tau)
        S[w] = q * scl[None, :]


# --------------------------------------------------------------------------------------------
# Propagation (src/AFQMC/SlaterDeterminantOperations/propagate.hpp)
# --------------------------------------------------------------------------------------------
def apply_expM(V, S, order=6, TA="N"):
    """S += sum_{n=1..order} (im V)^n / n! S, iteratively T_n = (im/n) V T_{n-1}
    (propagate.hpp:41-70).  In place on S [W,M,N]."""
    im = 1j if TA in "NT" else -1j
    T1 = S.copy()
    for n in range(1, order + 1):
        fact = im * (1.0 / float(n))
        if TA == "N":
            T2 = fact * np.matmul(V, T1)
        elif TA == "T":
            T2 = fact * np.matmul(np.swapaxes(V, 1, 2), T1)
        else:
            T2 = fact * np.matmul(np.conj(np.swapaxes(V, 1, 2)), T1)
        S += T2
        T1 = T2


def propagate_impl(S, P1, V, order=6, TA="N"):
    """S <- P1 exp(im V) P1 S (propagate.hpp:238-298), npol=1, dense V [W,M,M]."""
    W, M, N = S.shape
    if N == 0:
        return
    TMN = np.matmul(P1, S)
    apply_expM(V, TMN, order, TA)
    S[...] = np.matmul(P1, TMN)


# --------------------------------------------------------------------------------------------
# Hamiltonian operations (src/AFQMC/HamiltonianOperations/Real3IndexFactorization.hpp)
# --------------------------------------------------------------------------------------------
class Real3IndexFactorization:
    """Real dense 3-index Cholesky HamiltonianOperations, single determinant, npol = 1.

    Construction restates RealDenseHamiltonian::getHamiltonianOperations
    (src/AFQMC/Hamiltonians/RealDenseHamiltonian.cpp:139-180) and half_rotate_hamiltonian
    (src/AFQMC/HamiltonianOperations/detail/one_body.hpp:124-153).

    Likn : real [nspin_H2, M, M, Nc];  hij : complex [nspin_H1, M, M];  PsiT : list over spin of
    complex [N_s, M].
    """

    def __init__(self, walker_type, M, nup, ndn, Likn, hij, E0, PsiT):
        self.walker_type = walker_type
        self.M, self.nup, self.ndn = M, nup, ndn
        self.Likn = np.asarray(Likn, dtype=np.float64)
        self.nCV = self.Likn.shape[3]
        self.hij = np.asarray(hij, dtype=np.complex128)
        self.E0 = float(E0)
        nspin = 2 if walker_type == COLLINEAR else 1
        nel = [nup, ndn if walker_type == COLLINEAR else 0]
        ns_h2 = self.Likn.shape[0]
        ns_h1 = self.hij.shape[0]
        # haj [nel_tot, M] = PsiT_s * h_s  (one_body.hpp:144-148)
        self.haj = np.zeros((nel[0] + nel[1], M), dtype=np.complex128)
        for s in range(nspin):
            if nel[s] == 0:
                continue
            self.haj[s * nel[0]:s * nel[0] + nel[s]] = PsiT[s] @ self.hij[s % ns_h1]
        # Lnak[s] [Nc, N_s, M]: Lnak[n,a,j] = sum_i PsiT[a,i] L[i,j,n]  (RealDenseHamiltonian.cpp:141-161)
        self.Lnak = []
        for s in range(nspin):
            Ls = self.Likn[s % ns_h2]
            if nel[s] == 0:
                self.Lnak.append(np.zeros((self.nCV, 0, M), dtype=np.complex128))
                continue
            PL = (PsiT[s] @ Ls.reshape(M, M * self.nCV)).reshape(nel[s], M, self.nCV)
            self.Lnak.append(np.ascontiguousarray(PL.transpose(2, 0, 1)))
        # v0[i,l] = -1/2 sum_{j,n} L[i,j,n] L[l,j,n]  (RealDenseHamiltonian.cpp:163-180)
        self.vexx = np.stack([-0.5 * (L.reshape(M, -1) @ L.reshape(M, -1).T) for L in self.Likn])

    def number_of_cholesky_vectors(self):
        return self.nCV

    # vbias (Real3IndexFactorization.hpp:328-428), ndet == 1 branch
    def vbias(self, G, dt):
        W = G.shape[0]
        a = math.sqrt(dt) * (2.0 if self.walker_type == CLOSED else 1.0)
        nel = self.nup + (self.ndn if self.walker_type == COLLINEAR else 0)
        G3 = G.reshape(W, nel, self.M)
        v = np.zeros((W, self.nCV), dtype=np.complex128)
        nspin = 2 if self.walker_type == COLLINEAR else 1
        for s in range(nspin):
            ns = self.nup if s == 0 else self.ndn
            if ns == 0:
                continue
            Gs = G3[:, s * self.nup:s * self.nup + ns, :]
            v += a * (Gs.reshape(W, -1) @ self.Lnak[s].reshape(self.nCV, -1).T)
        return v

    # vHS (Real3IndexFactorization.hpp:282-326): [nspin_vHS, W, M, M]
    def vHS(self, X, dt):
        a = math.sqrt(dt)
        nst = self.Likn.shape[0] if self.walker_type == COLLINEAR else 1
        M = self.M
        out = []
        for s in range(nst):
            Lt = self.Likn[s].reshape(M * M, self.nCV).T  # real L, complex X
            V = (X.real @ Lt) + 1j * (X.imag @ Lt)
            out.append(a * V.reshape(-1, M, M))
        return np.stack(out)

    # energy (Real3IndexFactorization.hpp:138-174) + energy_impl (476-590)
    def energy(self, G, addH1=True, addEJ=True, addEXX=True):
        W = G.shape[0]
        nspin = 2 if self.walker_type == COLLINEAR else 1
        nel = self.nup + (self.ndn if self.walker_type == COLLINEAR else 0)
        G3 = G.reshape(W, nel, self.M)
        E = np.zeros((W, 3), dtype=np.complex128)
        if addH1:
            E[:, 0] = self.E0
        Kl = np.zeros((W, self.nCV), dtype=np.complex128)
        scl = 2.0 if self.walker_type == CLOSED else 1.0
        for s in range(nspin):
            ns = self.nup if s == 0 else self.ndn
            if ns == 0:
                continue
            Gs = G3[:, s * self.nup:s * self.nup + ns, :]
            if addH1:
                E[:, 0] += scl * np.einsum("waj,aj->w", Gs, self.haj[s * self.nup:s * self.nup + ns])
            if addEXX:
                for w in range(W):
                    # Twbna = sum_k G[w,b,k] Lnak[n,a,k]
                    T = (Gs[w] @ self.Lnak[s].reshape(self.nCV * ns, self.M).T).reshape(
                        ns, self.nCV, ns)
                    E[w, 1] += -0.5 * scl * np.sum(T * T.transpose(2, 1, 0))
                    if addEJ:
                        Kl[w] += np.einsum("ana->n", T)
        if addEJ:
            sclj = 4.0 if self.walker_type == CLOSED else 1.0
            E[:, 2] += 0.5 * sclj * np.einsum("wn,wn->w", Kl, Kl)
        return E

    # getOneBodyPropagatorMatrix (Real3IndexFactorization.hpp:99-124) + add_one_body_shifts
    # (one_body.hpp:65-85): H1 = dt*h + dt*v0 + vHS(vMF, dt)
    def getOneBodyPropagatorMatrix(self, dt, vMF):
        nspin = 2 if self.walker_type == COLLINEAR else 1
        mf = self.vHS(vMF[None, :], dt)[:, 0]  # [nst, M, M]
        H1 = np.zeros((nspin, self.M, self.M), dtype=np.complex128)
        for s in range(nspin):
            H1[s] = dt * self.hij[s % self.hij.shape[0]]
            H1[s] += dt * self.vexx[s % self.vexx.shape[0]] + mf[s % mf.shape[0]]
        return H1


# --------------------------------------------------------------------------------------------
# Single-determinant NOMSD trial (src/AFQMC/Wavefunctions/NOMSD.{hpp,cpp})
# --------------------------------------------------------------------------------------------
class NOMSD:
    def __init__(self, ham: Real3IndexFactorization, PsiT, ci=1.0 + 0j):
        self.ham = ham
        self.PsiT = [np.asarray(p, dtype=np.complex128) for p in PsiT]
        self.ci = complex(ci)
        self.walker_type = ham.walker_type
        self.M, self.nup, self.ndn = ham.M, ham.nup, ham.ndn

    def _log_ci(self):
        return np.log(complex(1e-12) if abs(self.ci) < 1e-12 else np.conj(self.ci))

    def DensityMatrix(self, SA, SB, compact=True):
        """NOMSD::DensityMatrix (NOMSD.hpp:293-343): returns (G [W, nel*M], ovlp)."""
        W = SA.shape[0]
        ov = np.zeros(W, dtype=np.complex128)
        GA = MixedDensityMatrix(self.PsiT[0], SA, ov, compact)
        if self.walker_type == CLOSED:
            ov *= 2.0
            G = GA.reshape(W, -1)
        else:
            GB = MixedDensityMatrix(self.PsiT[1], SB, ov, compact)
            G = np.concatenate([GA.reshape(W, -1), GB.reshape(W, -1)], axis=1)
        return G, ov

    def vbias(self, SA, SB, dt):
        """NOMSD::vbias (NOMSD.cpp:39-61)."""
        G, _ = self.DensityMatrix(SA, SB)
        return self.ham.vbias(G, dt)

    def Energy(self, SA, SB):
        """NOMSD::Energy, ndet == 1 (NOMSD.cpp:159-182): (E [W,3], Ov [W])."""
        G, ov = self.DensityMatrix(SA, SB)
        E = self.ham.energy(G)
        return E, ov + self._log_ci()

    def Log_Overlap(self, SA, SB):
        """NOMSD::Log_Overlap, ndet == 1 (NOMSD.cpp:280-301)."""
        ov = np.zeros(SA.shape[0], dtype=np.complex128)
        Log_Overlap(self.PsiT[0], SA, ov)
        if self.walker_type == CLOSED:
            ov *= 2.0
        else:
            Log_Overlap(self.PsiT[1], SB, ov)
        return ov + self._log_ci()

    def vMF(self, dt):
        """NOMSD::vMF, ndet == 1 (NOMSD.cpp:437-465): vbias of the trial's own G."""
        PsiA = self.PsiT[0].conj().T[None]
        ov = np.zeros(1, dtype=np.complex128)
        G = MixedDensityMatrix(self.PsiT[0], PsiA, ov).reshape(1, -1)
        if self.walker_type == COLLINEAR:
            PsiB = self.PsiT[1].conj().T[None]
            GB = MixedDensityMatrix(self.PsiT[1], PsiB, ov).reshape(1, -1)
            G = np.concatenate([G, GB], axis=1)
        return self.ham.vbias(G, dt)[0]

    def initial_walker(self):
        """Every walker starts as the trial (NOMSD.cpp:131-153): S = PsiT^H."""
        SA = self.PsiT[0].conj().T
        SB = self.PsiT[1].conj().T if self.walker_type == COLLINEAR else None
        return SA, SB


# --------------------------------------------------------------------------------------------
# Force-bias fields (src/AFQMC/Utilities/probit.h, Propagators/construct_X_kernel.hpp)
# --------------------------------------------------------------------------------------------
_PA = [-3.969683028665376e+01, 2.209460984245205e+02, -2.759285104469687e+02,
       1.383577518672690e+02, -3.066479806614716e+01, 2.506628277459239e+00]
_PB = [-5.447609879822406e+01, 1.615858368580409e+02, -1.556989798598866e+02,
       6.680131188771972e+01, -1.328068155288572e+01]
_PC = [-7.784894002430293e-03, -3.223964580411365e-01, -2.400758277161838e+00,
       -2.549732539343734e+00, 4.374664141464968e+00, 2.938163982698783e+00]
_PD = [7.784695709041462e-03, 3.224671290700398e-01, 2.445134137142996e+00,
       3.754408661907416e+00]


def probit(p: np.ndarray) -> np.ndarray:
    """Acklam's rational approximation of the inverse normal CDF (probit.h:57-135)."""
    p = np.asarray(p, dtype=np.float64)
    out = np.zeros_like(p)
    lo = (p > 0) & (p < 0.02425)
    hi = (p > 0.97575) & (p < 1)
    mid = (p >= 0.02425) & (p <= 0.97575)
    if np.any(lo):
        q = np.sqrt(-2 * np.log(p[lo]))
        out[lo] = ((((((_PC[0] * q + _PC[1]) * q + _PC[2]) * q + _PC[3]) * q + _PC[4]) * q + _PC[5])
                   / ((((_PD[0] * q + _PD[1]) * q + _PD[2]) * q + _PD[3]) * q + 1))
    if np.any(hi):
        q = np.sqrt(-2 * np.log(1 - p[hi]))
        out[hi] = -((((((_PC[0] * q + _PC[1]) * q + _PC[2]) * q + _PC[3]) * q + _PC[4]) * q + _PC[5])
                    / ((((_PD[0] * q + _PD[1]) * q + _PD[2]) * q + _PD[3]) * q + 1))
    if np.any(mid):
        q = p[mid] - 0.5
        r = q * q
        out[mid] = ((((((_PA[0] * r + _PA[1]) * r + _PA[2]) * r + _PA[3]) * r + _PA[4]) * r + _PA[5]) * q
                    / (((((_PB[0] * r + _PB[1]) * r + _PB[2]) * r + _PB[3]) * r + _PB[4]) * r + 1))
    out[p == 0] = -np.inf
    out[p == 1] = np.inf
    return out


def construct_X(vbias, u, vMF, vbias_bound):
    """construct_X_impl, continuous charge fields, no projection, not free projection
    (construct_X_kernel.hpp:20-89).  Returns (X [W,Nc], HW [W])."""
    def clamp(z):
        a = np.abs(z)
        return np.where(a > vbias_bound, z / np.where(a == 0, 1, a) * vbias_bound, z)
    vmf_t = clamp(vMF)[None, :]
    vb_t = clamp(vbias)
    vdiff = 1j * (vb_t - vmf_t)
    X = probit(u) + vdiff
    HW = np.sum(-vdiff * (X - 0.5 * vdiff), axis=1)
    return X, HW


def meanfield_factor(X, vMF):
    """mf[w] = -0.5 Re(vMF.vMF) + im * sum_n X[w,n] vMF[n] (AFQMCBasePropagator.cpp:334-336)."""
    return -0.5 * np.dot(vMF, vMF).real + 1j * (X @ vMF)


# --------------------------------------------------------------------------------------------
# Phaseless update (src/AFQMC/Propagators/WalkerSetUpdate.hpp)
# --------------------------------------------------------------------------------------------
@dataclass
class BoundStats:
    total: int = 0
    upper: int = 0
    lower: int = 0


def walker_update(props, new_ovlp, mf, hw, dt, Eshift, E0, lower_cut, upper_cut, stats=None):
    """Hybrid, phaseless, no CP constraint (WalkerSetUpdate.hpp:46-58, 69-191).
    props: complex [W, 11] walker scalars, updated in place."""
    stats = stats if stats is not None else BoundStats()
    W = props.shape[0]
    hi = Eshift + upper_cut * math.sqrt(2.0 / dt)
    lo = Eshift - lower_cut * math.sqrt(2.0 / dt)
    for i in range(W):
        old_ov = complex(props[i, OVLP])
        old_el = complex(props[i, PSEUDO_ELOC])
        dth = new_ovlp[i].imag - old_ov.imag - mf[i].imag
        scale = max(0.0, math.cos(dth))
        props[i, THETA] = dth
        eloc = (mf[i] - hw[i] - (new_ovlp[i] - old_ov)) / dt + E0
        if not math.isfinite(eloc.real):
            props[i, WEIGHT] = 0.0
            props[i, PHASE] = 0.0
            eloc = old_el
        else:
            stats.total += 1
            if eloc.real > hi:
                stats.upper += 1
            elif eloc.real < lo:
                stats.lower += 1
            eloc = complex(min(max(eloc.real, lo), hi), eloc.imag)
            w = np.exp(-dt * (eloc - Eshift))
            props[i, WEIGHT] *= scale * abs(w)
            props[i, PHASE] *= w / abs(w)
        props[i, PSEUDO_ELOC] = eloc
        props[i, OVLP] = new_ovlp[i]


def bound_walker_weights(props, floor, fraction, target_pop, stats=None):
    """(WalkerSetUpdate.hpp:198-218)"""
    stats = stats if stats is not None else BoundStats()
    mx = max(floor, fraction * target_pop)
    for i in range(props.shape[0]):
        a = abs(props[i, WEIGHT])
        stats.total += 1
        if a > mx:
            stats.upper += 1
            props[i, WEIGHT] *= mx / a


# --------------------------------------------------------------------------------------------
# One-body propagator (AFQMCBasePropagator.cpp:42-214, numerics/operations/exp.hpp:27-60)
# --------------------------------------------------------------------------------------------
def hermitize(A):
    """(numerics/operations/tensor.hpp:75-93)"""
    A = A.copy()
    n = A.shape[-1]
    for i in range(n):
        A[..., i, i] = A[..., i, i].real
        for j in range(i + 1, n):
            A[..., i, j] = 0.5 * A[..., i, j] + 0.5 * np.conj(A[..., j, i])
            A[..., j, i] = np.conj(A[..., i, j])
    return A


def exp_hermitian(A):
    """exp(A) = M exp(V) M^H via eigh (exp.hpp:27-60)."""
    V, Mv = np.linalg.eigh(A)
    Ms = Mv * np.sqrt(np.exp(V))[None, :]
    return Ms @ Ms.conj().T


def truncate_like_csr(P, vcut=1e-8):
    """to_csr keeps |x| > vcut (numerics/sparse/csr_utils.hpp:43-67)."""
    return np.where(np.abs(P) > vcut, P, 0)


def generateP1(wfn: NOMSD, dt, denseP1=False):
    """vMF (zero imag), H1, hermitize, x(-1/2), exp; CSR truncation unless denseP1; a P1 that is
    real to 1e-14 is applied as its real part (the host path's real CSR, cpp:142-207).
    Returns (P1 [nspin,M,M], vMF [Nc])."""
    vMF = wfn.vMF(dt).real.astype(np.complex128)  # math::zero_imag
    H1 = wfn.ham.getOneBodyPropagatorMatrix(dt, vMF)
    H1 = hermitize(H1) * (-0.5)
    P = np.stack([exp_hermitian(h) for h in H1])
    if not denseP1:
        vals = P[np.abs(P) > 1e-8]
        real = np.max(np.abs(vals.imag)) <= 1e-14 * np.max(np.abs(vals))
        P = truncate_like_csr(P.real if real else P).astype(np.complex128)
    return P, vMF


# --------------------------------------------------------------------------------------------
# The propagator and the driver loop
# --------------------------------------------------------------------------------------------
@dataclass
class PropagatorParams:
    """PropagatorParameters defaults for a non-model Hamiltonian (parameters.hpp:103-131,
    parameter_defaults.cpp:274-289)."""
    dt: float = 0.01
    taylor_n: int = 6
    vbias_bound: float = 50.0
    upper_cutoff_scale: float = 10.0
    lower_cutoff_scale: float = 1.0
    weight_bound_floor: float = 100.0
    weight_bound_fraction: float = 0.1
    denseP1: bool = False


@dataclass
class WalkerSet:
    """Walker rows split into S blocks and the 11 scalar properties (WalkerSetBase.cpp:44-125)."""
    SA: np.ndarray
    SB: np.ndarray | None
    props: np.ndarray
    target_pop: int
    walker_type: int = CLOSED

    @staticmethod
    def from_trial(wfn: NOMSD, W: int):
        SA0, SB0 = wfn.initial_walker()
        SA = np.repeat(SA0[None], W, axis=0).astype(np.complex128)
        SB = np.repeat(SB0[None], W, axis=0).astype(np.complex128) if SB0 is not None else None
        props = np.zeros((W, NPROP), dtype=np.complex128)
        props[:, WEIGHT] = 1.0
        props[:, PHASE] = 1.0
        return WalkerSet(SA, SB, props, W, wfn.walker_type)


class Propagator:
    """AFQMCBasePropagator, hybrid force-bias, dense vHS (AFQMCBasePropagator.cpp:289-392)."""

    def __init__(self, wfn: NOMSD, params: PropagatorParams):
        self.wfn = wfn
        self.p = params
        self.P1, self.vMF = generateP1(wfn, params.dt, params.denseP1)
        self.eloc_stats = BoundStats()
        self.weight_stats = BoundStats()
        self.last = {}

    def propagate(self, ws: WalkerSet, Eshift, u):
        """One step.  u: uniforms [W, Nc] (the field RNG block, rng_block_size = Nc)."""
        dt = self.p.dt
        wfn = self.wfn
        vb = wfn.vbias(ws.SA, ws.SB, dt)
        X, HW = construct_X(vb, u, self.vMF, self.p.vbias_bound)
        mf = meanfield_factor(X, self.vMF)
        V = wfn.ham.vHS(X, dt)
        propagate_impl(ws.SA, self.P1[0], V[0], self.p.taylor_n)
        if ws.walker_type == COLLINEAR:
            propagate_impl(ws.SB, self.P1[1 % self.P1.shape[0]], V[1 % V.shape[0]], self.p.taylor_n)
        new_ov = wfn.Log_Overlap(ws.SA, ws.SB)
        self.last = dict(vbias=vb, X=X, HW=HW, mf=mf, new_ov=new_ov)
        walker_update(ws.props, new_ov, mf, HW, dt, Eshift, wfn.ham.E0,
                      self.p.lower_cutoff_scale, self.p.upper_cutoff_scale, self.eloc_stats)
        bound_walker_weights(ws.props, self.p.weight_bound_floor, self.p.weight_bound_fraction,
                             ws.target_pop, self.weight_stats)

    def orthogonalize(self, ws: WalkerSet):
        """(AFQMCBasePropagator.cpp:735-741; orthogonalize.hpp:442-469)"""
        ldet = np.zeros(ws.SA.shape[0], dtype=np.complex128)
        orthogonalize(ws.SA, ldet)
        if ws.walker_type == COLLINEAR:
            orthogonalize(ws.SB, ldet)
        ws.props[:, OVLP] = self.wfn.Log_Overlap(ws.SA, ws.SB)
        return ldet


def population_control_single_rank(rng: HostRandomGenerator, ws: WalkerSet):
    """population_control on one rank (population_control.hpp:218-255)."""
    absw = np.abs(ws.props[:, WEIGHT])
    off = comb(rng, absw, absw.size)
    src = single_rank_slot_map(off)
    ws.SA[...] = ws.SA[src]
    if ws.SB is not None:
        ws.SB[...] = ws.SB[src]
    ws.props[...] = ws.props[src]
    w = ws.props[:, WEIGHT]
    ws.props[:, WEIGHT] = w / np.abs(w)
    return off


def energy_measure(wfn: NOMSD, ws: WalkerSet):
    """EnergyEstimator::measure (EnergyEstimator.h:51-100): weighted sums of E1, EXX, EJ."""
    E, ov = wfn.Energy(ws.SA, ws.SB)
    w = ws.props[:, WEIGHT]
    avg = E.T @ w
    return dict(E=E, ovlp=ov, numerator=avg, denominator=np.sum(w),
                energy=(np.sum(avg) / np.sum(w)).real)


def average_pseudo_energy(ws: WalkerSet, dt):
    """averagePseudoEnergy (Drivers/average_energy.hpp:53-63)."""
    w = ws.props[:, WEIGHT]
    e = np.exp(dt * ws.props[:, PSEUDO_ELOC])
    return (math.log((np.sum(w * e) / np.sum(w)).real)) / dt


def average_energy(ws: WalkerSet):
    """averageEnergy (Drivers/average_energy.hpp:67-76)."""
    w = ws.props[:, WEIGHT]
    e = ws.props[:, E1] + ws.props[:, EXX] + ws.props[:, EJ]
    return (np.sum(w * e) / np.sum(w)).real


@dataclass
class RunParams:
    steps: int = 400
    walker_ortho_interval: int = 5
    population_control_interval: int = 10
    measure_interval: int = 10
    equilibration_steps: int = 100
    seed: int = 0


def run_afqmc(wfn: NOMSD, prop: Propagator, ws: WalkerSet, rp: RunParams, field_uniforms=None,
              on_step=None):
    """execute_simulation initialisation (execute.cpp:124-184) + run_afqmc loop
    (Drivers/run_afqmc.cpp:69-113).  field_uniforms(step) may override the field RNG draws."""
    walker_rng = HostRandomGenerator(split_seed(rp.seed, 0, 0))
    field_rng = HostRandomGenerator(split_seed(rp.seed, 0, 1))
    E, ov = wfn.Energy(ws.SA, ws.SB)
    ws.props[:, OVLP] = ov
    ws.props[:, E1], ws.props[:, EXX], ws.props[:, EJ] = E[:, 0], E[:, 1], E[:, 2]
    ws.props[:, PSEUDO_ELOC] = E[:, 0] + E[:, 1] + E[:, 2]
    Eshift = average_energy(ws)
    # Propagator construction comes after the initial energy (execute.cpp:188-192)
    f = 1 - math.exp(-10.0 / rp.equilibration_steps) if rp.equilibration_steps > 1 else 1.0
    W, Nc = ws.SA.shape[0], wfn.ham.nCV
    energies = []
    for step in range(rp.steps):
        if field_uniforms is not None:
            u = field_uniforms(step)
        else:
            u = field_rng.sample_uniform(W * Nc).reshape(W, Nc)
        prop.propagate(ws, Eshift, u)
        if step % rp.walker_ortho_interval == 0:
            prop.orthogonalize(ws)
        if step % rp.population_control_interval == 0:
            population_control_single_rank(walker_rng, ws)
        if step >= rp.equilibration_steps:
            if step % rp.measure_interval == 0:
                energies.append((step, energy_measure(wfn, ws)["energy"]))
        else:
            Eshift += f * (average_pseudo_energy(ws, prop.p.dt) - Eshift)
        if on_step is not None:
            on_step(step, ws, Eshift)
    return energies, Eshift


def full_g_vbias(Likn, G, dt, walker_type):
    """Real3IndexFactorization::vbias on a full density matrix G [nspin][M][M]
    (Real3IndexFactorization.hpp:389-427): a sum_s sum_{ik} L_s[i][k][n] G_s[i][k], with
    a = sqrt(dt) (2 sqrt(dt) for CLOSED)."""
    L = np.asarray(Likn)
    a = math.sqrt(dt) * (2.0 if walker_type == CLOSED else 1.0)
    return a * sum(np.einsum("ikn,ik->n", L[s % L.shape[0]], G[s]) for s in range(G.shape[0]))


def onerdm(wfn: NOMSD, ws: WalkerSet):
    """The MixedEstimator's OneRDM, single reference (Estimators/Observables/onerdm.hpp:39-64,
    MixedEstimator.hpp:42-108): sum_w w_w G_w per spin block with the full mixed density matrix
    G_w = (S_w (PsiT S_w)^{-1} PsiT)^T (density_matrix.hpp:535-601, compact = false)."""
    blocks = [ws.SA] if ws.walker_type != COLLINEAR else [ws.SA, ws.SB]
    out = []
    off = 0
    for S in blocks:
        N = S.shape[2]
        PsiT = wfn.PsiT[0][off:off + N] if len(wfn.PsiT) == 1 else wfn.PsiT[len(out)]
        acc = np.zeros((S.shape[1], S.shape[1]), complex)
        for w in range(S.shape[0]):
            Mf = S[w] @ np.linalg.inv(PsiT @ S[w]) @ PsiT
            acc += ws.props[w, WEIGHT] * Mf.T
        out.append(acc)
        off += N
    return np.stack(out)



class NOMSDMulti:
    """NOMSD with several determinants (NOMSD.cpp:93-333, 159-217; Real3IndexFactorization.hpp
    :389-427): hams[d] built with determinant d's PsiT, coefficients ci.  vMF is given (the
    pairwise several-determinant vMF, NOMSD.cpp:466-520, is the caller's)."""

    def __init__(self, hams, PsiTs, ci, vMF=None):
        self.hams = list(hams)
        self.ham = self.hams[0]
        self.PsiTs = [[np.asarray(p, np.complex128) for p in P] for P in PsiTs]
        self.ci = np.asarray(ci, np.complex128)
        self.walker_type = self.ham.walker_type
        self.M, self.nup, self.ndn = self.ham.M, self.ham.nup, self.ham.ndn
        self._vMF = None if vMF is None else np.asarray(vMF, np.complex128)

    def _per_det(self, SA, SB, compact=True):
        out = []
        for d, P in enumerate(self.PsiTs):
            out.append(NOMSD(self.hams[d], P).DensityMatrix(SA, SB, compact))
        return out

    def Log_Overlap(self, SA, SB):
        lo = []
        for d, P in enumerate(self.PsiTs):
            ov = np.zeros(SA.shape[0], complex)
            Log_Overlap(P[0], SA, ov)
            if self.walker_type == CLOSED:
                ov *= 2.0
            else:
                Log_Overlap(P[1], SB, ov)
            c = self.ci[d]
            lo.append(ov + np.log(complex(1e-12) if abs(c) < 1e-12 else np.conj(c)))
        lo = np.array(lo)
        m = lo[np.argmax(lo.real, axis=0), np.arange(lo.shape[1])]
        return m + np.log(np.sum(np.exp(lo - m), axis=0))

    def Energy(self, SA, SB):
        Ed, ov = [], []
        for d, P in enumerate(self.PsiTs):
            G, o = NOMSD(self.hams[d], P).DensityMatrix(SA, SB)
            Ed.append(self.hams[d].energy(G))
            ov.append(o)
        Ed, ov = np.array(Ed), np.array(ov)
        m = ov[np.argmax(ov.real, axis=0), np.arange(ov.shape[1])]
        f = np.conj(self.ci)[:, None] * np.exp(ov - m)
        E = np.einsum("dw,dwq->wq", f, Ed) / f.sum(0)[:, None]
        return E, np.log(f.sum(0)) + m

    def initial_walker(self):
        """NOMSD::initial_guess (NOMSD.cpp:132-153): the determinant with the largest |c|."""
        d = int(np.argmax(np.abs(self.ci)))
        P = self.PsiTs[d]
        return P[0].conj().T.copy(), (P[1].conj().T.copy() if self.walker_type == COLLINEAR
                                      else None)

    def MixedDensityMatrix(self, SA, SB, log_m):
        """Full G [W, nspin, M, M] and the reference's Ov (linear sum + log_m)."""
        W = SA.shape[0]
        nspin = 2 if self.walker_type == COLLINEAR else 1
        G = np.zeros((W, nspin, self.M, self.M), complex)
        Ov = np.zeros(W, complex)
        for d, P in enumerate(self.PsiTs):
            ot = np.zeros(W, complex)
            Gs = [MixedDensityMatrix(P[0], SA, ot, compact=False)]
            if self.walker_type == CLOSED:
                ot *= 2.0
            else:
                Gs.append(MixedDensityMatrix(P[1], SB, ot, compact=False))
            wd = np.conj(self.ci[d]) * np.exp(ot - log_m)
            G += wd[:, None, None, None] * np.stack(Gs, 1)
            Ov += wd
        return G / Ov[:, None, None, None], Ov + log_m

    def vbias(self, SA, SB, dt):
        """Full-G branch of Real3IndexFactorization::vbias (hpp:389-427); the weights' shift
        cancels in G, so the walkers' own log overlap serves."""
        G, _ = self.MixedDensityMatrix(SA, SB, self.Log_Overlap(SA, SB))
        a = math.sqrt(dt) * (2.0 if self.walker_type == CLOSED else 1.0)
        L = self.ham.Likn  # [nspin_H2][M][M][Nc]
        v = np.zeros((SA.shape[0], L.shape[3]), complex)
        for s in range(G.shape[1]):
            v += a * np.einsum("ikn,wik->wn", L[s % L.shape[0]], G[:, s])
        return v

    def vMF(self, dt):
        return self._vMF.copy()
