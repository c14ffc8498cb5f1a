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
