"""ORACLE — test infrastructure only: back-propagation restated in numpy.

AFQMCBasePropagator::BackPropagate (Propagators/AFQMCBasePropagator.cpp:403-533): the trial,
one copy per walker in the walker layout (PsiT^H [M][N] per spin), is propagated backwards
through the stored fields of the last nbp steps, newest first, with apply_propagators<'H'>:
S <- P1^H sum_n (-i V^H)^n / n! P1^H S (propagate.hpp:41-70, 238-298), V = vHS(X) of that step,
and a QR re-orthogonalisation (orthogonalize.hpp:131-169) whenever ni % nstab == 0 and at the
last step (ni == 0), its log det accumulated into logdetR.

BackPropEstimator (Estimators/BackPropEstimator.hpp:36-120, 170-235) with one reference: the
walkers' weights times the path-restoration factors of the last nbp steps
(WalkerSetUpdate.hpp:128-147: w / |w| / max(0, cos dtheta), zero where the projection or a
non-finite energy killed the walker), and the full density matrix between the back-propagated
trial (bra, batched A: T = A^H B) and the walker stored at the start of the window,
G = (B T^-1 A^H)^T (density_matrix.hpp:603-650).  With one reference the overlap factor
conj(c) e^{log ov} / sum over references is 1.  OneRDM (Observables/onerdm.hpp) accumulates
sum_w weight_w G_w, and the measurement divides by sum_w weight_w (Measurements.hpp:96-123).
"""
import numpy as np

from oracle.afqmc import apply_expM, orthogonalize


def back_propagate(refs, P1, V_hist, order, nstab):
    """refs: per spin [W][M][N_s] (copies of the trial, modified in place); P1 per spin [M][M];
    V_hist: vHS of the stored steps, oldest first, each [nst][W][M][M] (nst 1 or 2); returns
    logdetR [W]."""
    W = refs[0].shape[0]
    logdetR = np.zeros(W, dtype=np.complex128)
    nbp = len(V_hist)
    for ni in range(nbp - 1, -1, -1):
        V = V_hist[ni]
        for s, S in enumerate(refs):
            if S.shape[2] == 0:
                continue
            Vs = V[s % V.shape[0]]
            P1h = P1[s % len(P1)].conj().T
            T = np.matmul(P1h, S)
            apply_expM(Vs, T, order, "H")
            S[...] = np.matmul(P1h, T)
        if ni == 0 or ni % nstab == 0:
            ld = np.zeros(W, dtype=np.complex128)
            for S in refs:
                if S.shape[2]:
                    orthogonalize(S, ld)
            logdetR += ld
    return logdetR


def path_restored_weights(weights, factors):
    """weights [W] times the product of the per-step factors [nbp][W]."""
    return np.asarray(weights, dtype=np.complex128) * np.prod(np.asarray(factors), axis=0)


def bp_onerdm(refs, anchors, weights):
    """sum_w weight_w G_w / sum_w weight_w, G_w = (B T^-1 A^H)^T per spin with A the
    back-propagated trial, B the anchored walker.  Returns [nspin][M][M]."""
    out = []
    for A, B in zip(refs, anchors):
        W, M, N = B.shape
        if N == 0:
            out.append(np.zeros((M, M), dtype=np.complex128))
            continue
        AH = np.conj(np.swapaxes(A, 1, 2))
        T = np.matmul(AH, B)
        G = np.swapaxes(np.matmul(B, np.matmul(np.linalg.inv(T), AH)), 1, 2)
        out.append(np.einsum("w,wik->ik", weights, G) / np.sum(weights))
    return np.array(out)


def weight_factors(props_before, props_after, phase_col, theta_col):
    """Per-step factors as WalkerSetUpdate.hpp:128-147 forms them, from the walker properties
    before and after the step: the phase factor w / |w| (new phase / old phase) over
    max(0, cos dtheta), zero where that scale is zero or the walker's phase was zeroed."""
    p0 = props_before[:, phase_col]
    p1 = props_after[:, phase_col]
    scale = np.maximum(0.0, np.cos(props_after[:, theta_col].real))
    ok = (scale > np.finfo(np.float64).tiny) & (p0 != 0)
    out = np.zeros(p0.shape, dtype=np.complex128)
    out[ok] = (p1[ok] / p0[ok]) / scale[ok]
    return out
