"""ORACLE — test infrastructure only (see oracle/__init__.py).

Restatement of the reference's particle-hole multi-Slater-determinant (PHMSD) energy kernels,
src/AFQMC/Wavefunctions/detail/phmsd_impl.hpp, host branches:
  ph_excited_2body_energy_dense_cholesky (lines 33-153) and ph_excited_1body_energy (156-193).

Layouts (C order, as the reference's nda arrays):
  iexcit [ndet][2][nex]  holes (electron indices into refc) then particles (active orbitals)
  refc   [nelec]         reference configuration (active orbital of every electron)
  Twina  [nw][nelec][nchol][nact]
  R      [nw][ndet][nex][nact]
  wgt    [ndet][nw]
"""
from __future__ import annotations

import numpy as np


def _occupations(iex_d, refc):
    """occps(i): the active orbital electron i occupies in determinant d (phmsd_impl.hpp:71-80)."""
    nex = iex_d.shape[1]
    occ = np.array(refc, dtype=np.int64).copy()
    for i in range(occ.size):
        for e in range(nex):
            if iex_d[0, e] == i:
                occ[i] = iex_d[1, e]
                break
    return occ


def ph_excited_2body_energy_dense_cholesky(iexcit, refc, Twina, R, wgt, EX=None, EJ=None):
    """Returns (EX [nw], EJ [nw], KE [ndet][nw][nchol]); EX, EJ accumulate onto the given arrays
    (EX -= 1/2 wgt eX, EJ += 1/2 wgt (sum Kn^2 - eJ0)) as phmsd_impl.hpp:141-142 does."""
    nw, ndet, nex, nact = R.shape
    nelec, nchol = Twina.shape[1], Twina.shape[2]
    iex = np.asarray(iexcit).reshape(ndet, 2, nex)
    EX = np.zeros(nw, complex) if EX is None else np.array(EX, complex)
    EJ = np.zeros(nw, complex) if EJ is None else np.array(EJ, complex)
    KE = np.zeros((ndet, nw, nchol), complex)
    for iw in range(nw):
        T = Twina[iw]
        # spin-diagonal J of the reference configuration (phmsd_impl.hpp:82-88)
        Fref = sum(T[i, :, refc[i]] for i in range(nelec))
        eJ0 = np.sum(Fref * Fref)
        for d in range(ndet):
            Rxa = R[iw, d]
            occ = _occupations(iex[d], refc)
            Kn = np.zeros(nchol, complex)
            eX = 0j
            for e1 in range(nex):
                ip = iex[d, 0, e1]
                Fn = T[ip] @ Rxa[e1]
                eX += np.sum(Fn * Fn)
                Kn += Fn
                for e2 in range(e1 + 1, nex):
                    iq = iex[d, 0, e2]
                    Fn = T[iq] @ Rxa[e1]
                    Fn1 = T[ip] @ Rxa[e2]
                    eX += 2.0 * np.sum(Fn * Fn1)
                for j in range(nelec):
                    Fa = T[j].T @ T[ip, :, occ[j]]
                    eX += 2.0 * np.sum(Fa * Rxa[e1])
            for i in range(nelec):
                Oi, ri = occ[i], refc[i]
                if Oi != ri:
                    eX += np.sum(T[i, :, Oi] * T[i, :, Oi]) - np.sum(T[i, :, ri] * T[i, :, ri])
                for j in range(i + 1, nelec):
                    Oj, rj = occ[j], refc[j]
                    if Oi != ri or Oj != rj:
                        eX += 2.0 * (np.sum(T[i, :, Oj] * T[j, :, Oi]) -
                                     np.sum(T[i, :, rj] * T[j, :, ri]))
            for i in range(nelec):
                Kn += T[i, :, occ[i]]
            KE[d, iw] = Kn
            EX[iw] -= 0.5 * wgt[d, iw] * eX
            EJ[iw] += 0.5 * wgt[d, iw] * (np.sum(Kn * Kn) - eJ0)
    return EX, EJ, KE


def ph_excited_1body_energy(iexcit, refc, S, R, wgt, E=None):
    """E[iw] += sum_d wgt[d][iw] sum_p (S[iw][ip] . R[iw][d][p] + S[iw][ip][particle_p]
    - S[iw][ip][refc[ip]])  (phmsd_impl.hpp:173-184).  S [nw][nelec][nact]."""
    nw, ndet, nex, nact = R.shape
    iex = np.asarray(iexcit).reshape(ndet, 2, nex)
    E = np.zeros(nw, complex) if E is None else np.array(E, complex)
    for iw in range(nw):
        for d in range(ndet):
            e_ = 0j
            for p in range(nex):
                ip = iex[d, 0, p]
                e_ += np.sum(S[iw, ip] * R[iw, d, p]) + S[iw, ip, iex[d, 1, p]] - S[iw, ip, refc[ip]]
            E[iw] += wgt[d, iw] * e_
    return E


def phmsd_log_overlap(trial, S_up, S_dn):
    """PHMSD::Log_Overlap (Wavefunctions/PHMSD.cpp:804-900) for COLLINEAR walkers:
    per spin Log_OverlapForWoodbury (density_matrix.hpp:487-532: TMN = A B, TNN = TMN[refc],
    log det TNN accumulated with log_determinant_from_getrf, QQ0 = TMN TNN^{-1}), the unique
    excitation overlaps det(QQ0[particles, holes]) (phmsd_helpers.hpp:111-193), then
    log(sum_k c_k ov_up[k] ov_dn[k]) + log_ov.  trial: safire_b200.synth.PHMSDTrial layout;
    S_s [W, M, N_s].  Returns (log overlap [W], [ov_up [nuniq_up, W], ov_dn [nuniq_dn, W]])."""
    from oracle.afqmc import _getrf_ref, _getri_or_zero_ref, log_det_from_getrf
    W = S_up.shape[0]
    log_ov = np.zeros(W, complex)
    ovs = []
    for s, S in ((0, S_up), (1, S_dn)):
        A = trial.orbmat[s]
        refc = trial.refc[s]
        TMN = np.einsum("am,wmn->wan", A, S)
        QQ0 = np.empty_like(TMN)
        for w in range(W):
            lu, piv1, info = _getrf_ref(TMN[w][refc, :])
            log_ov[w] = log_det_from_getrf(lu, piv1, complex(log_ov[w]))
            QQ0[w] = TMN[w] @ _getri_or_zero_ref(lu, piv1)
        ov = [np.ones(W, complex)]
        for n in sorted(trial.exc[s]):
            for e in trial.exc[s][n]:
                holes, parts = e[:n], e[n:]
                ov.append(np.linalg.det(QQ0[:, parts][:, :, holes]))
        ovs.append(np.array(ov))
    tot = np.einsum("k,kw,kw->w", trial.coef, ovs[0][trial.det_up], ovs[1][trial.det_dn])
    return np.log(tot) + log_ov, ovs


# --------------------------------------------------------------------------------------------
# PHMSD energy (Wavefunctions/PHMSD.cpp:376-546 energy_alg1, COLLINEAR) and its building blocks
# --------------------------------------------------------------------------------------------
class ActiveSpaceHamiltonian:
    """Real3IndexFactorization tensors half-rotated with the active orbitals of a PHMSD trial
    (the HamiltonianOperations built for a PHMSD wavefunction: its 'nup/ndown' rows are the
    active orbitals, Real3IndexFactorization.hpp:598-602).  Lnak[s] [Nc][nact_s][M],
    haj[s] [nact_s][M]."""

    def __init__(self, trial, Likn, hij, E0):
        Likn = np.asarray(Likn, dtype=np.float64)
        hij = np.asarray(hij, dtype=np.complex128)
        M = trial.M
        self.E0 = float(E0)
        self.nCV = Likn.shape[3]
        self.Lnak, self.haj = [], []
        for s in (0, 1):
            A = trial.orbmat[s]
            L = Likn[s % Likn.shape[0]]
            PL = (A @ L.reshape(M, M * self.nCV)).reshape(A.shape[0], M, self.nCV)
            self.Lnak.append(np.ascontiguousarray(PL.transpose(2, 0, 1)))
            self.haj.append(A @ hij[s % hij.shape[0]])


def mixed_density_matrix_for_woodbury(A, S, refc):
    """det_ops::MixedDensityMatrixForWoodbury, compact (density_matrix.hpp:651-717):
    TAB = A S, TNN = TAB[refc], log det (getrf conventions), inverse, QQ0 = TAB TNN^{-1},
    G = TNN^{-T} S^T.  Returns (G [W,N,M], log_ov [W], QQ0 [W,nact,N])."""
    from oracle.afqmc import _getrf_ref, _getri_or_zero_ref, log_det_from_getrf
    W = S.shape[0]
    TAB = np.einsum("am,wmn->wan", A, S)
    G = np.empty((W, S.shape[2], S.shape[1]), complex)
    QQ0 = np.empty_like(TAB)
    logov = np.zeros(W, complex)
    for w in range(W):
        lu, piv1, info = _getrf_ref(TAB[w][refc, :])
        logov[w] = log_det_from_getrf(lu, piv1, 0j)
        inv = _getri_or_zero_ref(lu, piv1)
        QQ0[w] = TAB[w] @ inv
        G[w] = inv.T @ S[w].T
    return G, logov, QQ0


def excitation_overlaps(trial, s, QQ0):
    """calculate_overlaps (phmsd_helpers.hpp:111-193): [nuniq, W], index 0 = reference."""
    W = QQ0.shape[0]
    ov = [np.ones(W, complex)]
    for n in sorted(trial.exc[s]):
        for e in trial.exc[s][n]:
            ov.append(np.linalg.det(QQ0[:, e[n:]][:, :, e[:n]]))
    return np.array(ov)


def compact_R(iexcit, refc, QQ0):
    """get_compact_ph_R_matrices (phmsd_helpers.hpp:311-398): R [W][ndet][nex][nact] from the
    inverse Q of each nex x nex excitation block: R[p][orb_i] -= Q[p][q] QQ0[part_q][i] for every
    electron i, R[p][orb(hole_q)] += Q[p][q], orb = the determinant's occupations."""
    W, nact, nel = QQ0.shape
    ndet, two_nex = iexcit.shape
    nex = two_nex // 2
    R = np.zeros((W, ndet, nex, nact), complex)
    for d in range(ndet):
        holes, parts = iexcit[d, :nex], iexcit[d, nex:]
        orbs = np.array(refc).copy()
        orbs[holes] = parts
        for w in range(W):
            Q = QQ0[w][np.ix_(parts, holes)]
            if abs(np.linalg.det(Q)) == 0.0:
                continue
            Qi = np.linalg.inv(Q)
            for p in range(nex):
                for q in range(nex):
                    R[w, d, p, orbs] -= Qi[p, q] * QQ0[w, parts[q], :]
                    R[w, d, p, orbs[holes[q]]] += Qi[p, q]
    return R


def ph_reference_energy(H, s, G, refc, alpha):
    """ph_reference_energy / ph_ref_energy_impl (Real3IndexFactorization.hpp:212-235, 598-696)
    for COLLINEAR walkers: returns (E [W,3], Kl [W,Nc], Swia [W,N,nact], Twina [W,N,Nc,nact]).
    E1 = (E0 if alpha) + sum_i Swia[i, refc_i]; EXX = -1/2 sum Twina[i,n,refc_j] Twina[j,n,refc_i];
    EJ = 1/2 Kl.Kl with Kl[n] = sum_i Twina[i,n,refc_i]."""
    W, N, M = G.shape
    Swia = np.einsum("wik,ak->wia", G, H.haj[s])
    Twina = np.einsum("wik,nak->wina", G, H.Lnak[s])
    E = np.zeros((W, 3), complex)
    if alpha:
        E[:, 0] = H.E0
    r = np.asarray(refc)
    E[:, 0] += np.einsum("wii->w", Swia[:, :, r])
    Tr = Twina[:, :, :, r]  # [W, i, n, j] with j over electrons
    E[:, 1] += -0.5 * np.einsum("winj,wjni->w", Tr, Tr)
    Kl = np.einsum("wini->wn", Tr)
    E[:, 2] += 0.5 * np.einsum("wn,wn->w", Kl, Kl)
    return E, Kl, Swia, Twina


def _shells(trial, s):
    """(first unique index, iexcit) per excitation number, in the unique-index order."""
    out, k = [], 1
    for n in sorted(trial.exc[s]):
        e = trial.exc[s][n]
        out.append((k, e))
        k += e.shape[0]
    return out


def _couple(trial, s, vec_other):
    """sum over determinants of spin s's unique index u: c_k vec_other[det_other[k]] (the
    OpSpinDetCouplings CSR products of energy_alg1)."""
    det_s = trial.det_up if s == 0 else trial.det_dn
    det_o = trial.det_dn if s == 0 else trial.det_up
    nu = trial.unique_count(s)
    out = np.zeros((nu,) + vec_other.shape[1:], complex)
    for k in range(trial.coef.size):
        out[det_s[k]] += trial.coef[k] * vec_other[det_o[k]]
    return out


def phmsd_energy(trial, H, S_up, S_dn):
    """PHMSD::energy_alg1 (PHMSD.cpp:376-546), COLLINEAR: returns (E [W,3], log overlap [W])."""
    W = S_up.shape[0]
    Gu, lu, Qu = mixed_density_matrix_for_woodbury(trial.orbmat[0], S_up, trial.refc[0])
    Gd, ld, Qd = mixed_density_matrix_for_woodbury(trial.orbmat[1], S_dn, trial.refc[1])
    log_ov = lu + ld
    ovu = excitation_overlaps(trial, 0, Qu)
    ovd = excitation_overlaps(trial, 1, Qd)
    E = np.zeros((W, 3), complex)
    # spin up: weights, Ov, reference energy, excited energies
    wgt = _couple(trial, 0, ovd)                   # [nu_up, W]
    Ov = np.sum(wgt * ovu, axis=0)
    wgt = wgt * ovu
    eloc, Kl_up, Swia, Twina = ph_reference_energy(H, 0, Gu, trial.refc[0], True)
    E += eloc * Ov[:, None]
    KEr = np.zeros((trial.unique_count(0), W, H.nCV), complex)
    KEr[0] = Kl_up
    el = np.zeros((W, 3), complex)
    for k0, iex in _shells(trial, 0):
        R = compact_R(iex, trial.refc[0], Qu)
        w = wgt[k0:k0 + iex.shape[0]]
        el[:, 0] = ph_excited_1body_energy(iex, trial.refc[0], Swia, R, w, el[:, 0])
        EX, EJ, KE = ph_excited_2body_energy_dense_cholesky(iex, trial.refc[0], Twina, R, w,
                                                            el[:, 1], el[:, 2])
        el[:, 1], el[:, 2] = EX, EJ
        KEr[k0:k0 + iex.shape[0]] = KE
    E += el
    KEr = KEr * ovu[:, :, None]
    KEd = _couple(trial, 1, KEr) * ovd[:, :, None]  # [nu_dn, W, Nc]
    # spin down
    wgt = _couple(trial, 1, ovu) * ovd
    eloc, Kl_dn, Swia, Twina = ph_reference_energy(H, 1, Gd, trial.refc[1], False)
    E += eloc * Ov[:, None]
    E[:, 2] += np.einsum("wn,wn->w", KEd[0], Kl_dn)
    el = np.zeros((W, 3), complex)
    for k0, iex in _shells(trial, 1):
        R = compact_R(iex, trial.refc[1], Qd)
        w = wgt[k0:k0 + iex.shape[0]]
        el[:, 0] = ph_excited_1body_energy(iex, trial.refc[1], Swia, R, w, el[:, 0])
        EX, EJ, KEl = ph_excited_2body_energy_dense_cholesky(iex, trial.refc[1], Twina, R, w,
                                                             el[:, 1], el[:, 2])
        el[:, 1], el[:, 2] = EX, EJ
        el[:, 2] += np.einsum("dwn,dwn->w", KEd[k0:k0 + iex.shape[0]], KEl)
    E += el
    E = E / Ov[:, None]
    return E, np.log(Ov) + log_ov


def calculate_R(trial, s, QQ0, wgt):
    """calculate_R (phmsd_helpers.hpp:200-309): R [W][N][nact] = sum over unique excitations u
    (index 0 the reference) of wgt[u][w] times the Woodbury R of u: identity on the determinant's
    occupations plus, on the hole rows, -Q[p][q] QQ0[part_q][i] at orbs(i) and +Q[p][q] at
    orbs(hole_q)."""
    W, nact, nel = QQ0.shape
    refc = np.asarray(trial.refc[s])
    R = np.zeros((W, nel, nact), complex)
    R[:, np.arange(nel), refc] += wgt[0][:, None]
    u = 1
    for n in sorted(trial.exc[s]):
        for e in trial.exc[s][n]:
            holes, parts = e[:n], e[n:]
            orbs = refc.copy()
            orbs[holes] = parts
            for w in range(W):
                Q = QQ0[w][np.ix_(parts, holes)]
                if abs(np.linalg.det(Q)) == 0.0:
                    continue
                Qi = np.linalg.inv(Q)
                wu = wgt[u][w]
                R[w, np.arange(nel), orbs] += wu
                for p in range(n):
                    for q in range(n):
                        R[w, holes[p], orbs] -= wu * Qi[p, q] * QQ0[w, parts[q], :]
                        R[w, holes[p], orbs[holes[q]]] += wu * Qi[p, q]
            u += 1
    return R


def phmsd_mixed_density_matrix(trial, S_up, S_dn):
    """PHMSD::MixedDensityMatrix, compact, COLLINEAR (PHMSD.cpp:684-795): G [W][nact_up +
    nact_dn][M] = (R_s^T G_s) / Ov per spin block, and the log overlap [W]."""
    Gu, lu, Qu = mixed_density_matrix_for_woodbury(trial.orbmat[0], S_up, trial.refc[0])
    Gd, ld, Qd = mixed_density_matrix_for_woodbury(trial.orbmat[1], S_dn, trial.refc[1])
    ovu = excitation_overlaps(trial, 0, Qu)
    ovd = excitation_overlaps(trial, 1, Qd)
    wgt = _couple(trial, 0, ovd)
    Ov = np.sum(wgt * ovu, axis=0)
    Ru = calculate_R(trial, 0, Qu, wgt * ovu)
    Rd = calculate_R(trial, 1, Qd, _couple(trial, 1, ovu) * ovd)
    G = np.concatenate([np.einsum("wia,wik->wak", Ru, Gu), np.einsum("wia,wik->wak", Rd, Gd)],
                       axis=1) / Ov[:, None, None]
    return G, np.log(Ov) + lu + ld


def phmsd_vbias(ham, G, dt, nact_up):
    """PHMSD::vbias over Real3IndexFactorization::vbias (PHMSD.cpp:54-72,
    Real3IndexFactorization.hpp:328-384), COLLINEAR: v [W][Nc] = sqrt(dt) sum_s Lnak_s . G_s
    with G [W][nact_up + nact_dn][M] the compact PHMSD density matrix."""
    Gs = (G[:, :nact_up, :], G[:, nact_up:, :])
    return np.sqrt(dt) * sum(np.einsum("nak,wak->wn", ham.Lnak[s], Gs[s]) for s in (0, 1))


class PHMSDWavefunction:
    """The PHMSD wavefunction as AFQMCBasePropagator uses it: vbias (PHMSD.cpp:54-72) from the
    multi-determinant density matrix and the active-space Lnak, Log_Overlap (804-900), vHS and the
    one-body propagator from `ham` (a COLLINEAR oracle.afqmc.Real3IndexFactorization), and a given
    mean field vMF [Nc] (PHMSD::vMF, PHMSD.cpp:1329-1572, is the caller's)."""

    def __init__(self, trial, ham, Likn, hij, vMF):
        from oracle.afqmc import COLLINEAR
        self.trial = trial
        self.ham = ham
        self.walker_type = COLLINEAR
        self.H = ActiveSpaceHamiltonian(trial, Likn, hij, ham.E0)
        self._vMF = np.asarray(vMF, dtype=np.complex128)

    def vbias(self, SA, SB, dt):
        G, _ = phmsd_mixed_density_matrix(self.trial, SA, SB)
        return phmsd_vbias(self.H, G, dt, self.trial.orbmat[0].shape[0])

    def Log_Overlap(self, SA, SB):
        return phmsd_log_overlap(self.trial, SA, SB)[0]

    def Energy(self, SA, SB):
        """(E [W,3], log overlap [W]) by energy_alg1."""
        return phmsd_energy(self.trial, self.H, SA, SB)

    def initial_walker(self):
        """PHMSD::initial_guess (PHMSD.hpp:284-302): the configuration of the determinant with
        the largest coefficient, its orbitals' conjugates as columns (configuration_orbitals,
        PHMSD.hpp:364-375), in the excitation order of the configuration."""
        t = self.trial
        k = int(np.argmax(np.abs(np.asarray(t.coef))))
        out = []
        for s, u in ((0, int(t.det_up[k])), (1, int(t.det_dn[k]))):
            conf = np.asarray(t.refc[s]).copy()
            if u > 0:
                pos = 1
                for n in sorted(t.exc[s]):
                    e = t.exc[s][n]
                    if u < pos + len(e):
                        ex = e[u - pos]
                        conf[ex[:n]] = ex[n:]
                        break
                    pos += len(e)
            out.append(np.conj(np.asarray(t.orbmat[s])[conf]).T.copy())
        return out[0], out[1]

    def vMF(self, dt):
        return self._vMF.copy()
