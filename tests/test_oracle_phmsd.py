"""The oracle's PHMSD energy kernels against the reference's golden values
(tests/test_phmsd_components.cpp:41-47, 113-118)."""
import numpy as np
import pytest

from oracle import phmsd as P
from tests.golden import phmsd_golden as g


def _approx(a, b):
    # utils::Approx (tests/test_common.hpp:384-438): relative 1e-8 with an absolute floor
    return abs(a - b) <= 1e-8 * max(1.0, abs(b))


@pytest.mark.parametrize("nex", [1, 2, 3, 4, 5])
def test_ph_excited_2body_energy_golden(nex):
    iexcit, refc, T, R, wgt = g.fixture(nex)
    EX, EJ, KE = P.ph_excited_2body_energy_dense_cholesky(iexcit, refc, T, R, wgt)
    assert _approx(EX[0], g.EXJ_REF[nex - 1, 0]), (EX[0], g.EXJ_REF[nex - 1, 0])
    assert _approx(EJ[0], g.EXJ_REF[nex - 1, 1]), (EJ[0], g.EXJ_REF[nex - 1, 1])
    assert KE.shape == (g.NDET, g.NW, g.NCHOL)


def test_ph_excited_1body_energy_by_loops():
    """1-body Woodbury energy against an element-by-element evaluation of the same sum."""
    rs = np.random.default_rng(3)
    nw, ndet, nex, nact, nelec = 2, 7, 3, 9, 4
    iexcit, refc, T, R, wgt = g.fixture(nex)
    iexcit = iexcit[:ndet].copy() % np.array([nelec] * nex + [nact] * nex)
    S = rs.standard_normal((nw, nelec, nact)) + 1j * rs.standard_normal((nw, nelec, nact))
    R = rs.standard_normal((nw, ndet, nex, nact)) + 1j * rs.standard_normal((nw, ndet, nex, nact))
    wgt = rs.standard_normal((ndet, nw)) + 1j * rs.standard_normal((ndet, nw))
    refc = np.arange(nelec, dtype=np.int32)
    E = P.ph_excited_1body_energy(iexcit, refc, S, R, wgt)
    ref = np.zeros(nw, complex)
    for w in range(nw):
        for d in range(ndet):
            for p in range(nex):
                ip, pa = iexcit[d, p], iexcit[d, nex + p]
                s = sum(S[w, ip, a] * R[w, d, p, a] for a in range(nact))
                ref[w] += wgt[d, w] * (s + S[w, ip, pa] - S[w, ip, refc[ip]])
    assert np.allclose(E, ref, rtol=1e-12, atol=1e-12)


def _small_trial(seed=1):
    from safire_b200.synth import make_hamiltonian, make_phmsd_trial
    h1, _ = make_hamiltonian(24, 2, 0.99, seed)
    _, C = np.linalg.eigh(h1)
    return make_phmsd_trial(24, 6, 5, C, nocc=4, nvirt=8, ndet=120, seed=seed)


def test_phmsd_log_overlap_woodbury_vs_full_determinants():
    """The Woodbury evaluation (reference block LU + excitation-block determinants) against the
    sum over full determinants sum_k c_k det(D_up,k^H S_up) det(D_dn,k^H S_dn)."""
    t = _small_trial()
    rs = np.random.default_rng(4)
    W = 3
    S_up = rs.standard_normal((W, t.M, t.nup)) + 1j * rs.standard_normal((W, t.M, t.nup))
    S_dn = rs.standard_normal((W, t.M, t.ndn)) + 1j * rs.standard_normal((W, t.M, t.ndn))
    logov, _ = P.phmsd_log_overlap(t, S_up, S_dn)
    # occupied active orbitals of every unique excitation (electron order kept)
    occ = []
    for s in (0, 1):
        lst = [t.refc[s].copy()]
        for n in sorted(t.exc[s]):
            for e in t.exc[s][n]:
                o = t.refc[s].copy()
                o[e[:n]] = e[n:]
                lst.append(o)
        occ.append(lst)
    for w in range(W):
        tot = 0j
        for k in range(t.coef.size):
            du = np.linalg.det(t.orbmat[0][occ[0][t.det_up[k]]] @ S_up[w])
            dd = np.linalg.det(t.orbmat[1][occ[1][t.det_dn[k]]] @ S_dn[w])
            tot += t.coef[k] * du * dd
        assert abs(np.exp(logov[w]) - tot) <= 1e-10 * abs(tot), (w, np.exp(logov[w]), tot)


def test_phmsd_energy_woodbury_vs_single_determinants():
    """energy_alg1's Woodbury evaluation against sum_k c_k ov_k E_k / sum_k c_k ov_k with every
    determinant's local energy from the single-determinant (NOMSD, COLLINEAR) oracle."""
    from oracle import afqmc as O
    from safire_b200.synth import make_hamiltonian, make_phmsd_trial
    M, nup, ndn, Nc = 16, 4, 3, 6
    h1, Likn = make_hamiltonian(M, Nc, 0.9, seed=3)
    _, C = np.linalg.eigh(h1)
    t = make_phmsd_trial(M, nup, ndn, C, nocc=3, nvirt=5, ndet=40, seed=3)
    hij = h1[None].astype(complex)
    H = P.ActiveSpaceHamiltonian(t, Likn[None], hij, 0.7)
    rs = np.random.default_rng(8)
    W = 3
    S_up = (rs.standard_normal((W, M, nup)) + 1j * rs.standard_normal((W, M, nup))) / 4
    S_dn = (rs.standard_normal((W, M, ndn)) + 1j * rs.standard_normal((W, M, ndn))) / 4
    E, logov = P.phmsd_energy(t, H, S_up, S_dn)
    # brute force over determinants
    occ = []
    for s in (0, 1):
        lst = [t.refc[s].copy()]
        for n in sorted(t.exc[s]):
            for e in t.exc[s][n]:
                o = t.refc[s].copy()
                o[e[:n]] = e[n:]
                lst.append(o)
        occ.append(lst)
    num = np.zeros((W, 3), complex)
    den = np.zeros(W, complex)
    for k in range(t.coef.size):
        Pu = t.orbmat[0][occ[0][t.det_up[k]]]
        Pd = t.orbmat[1][occ[1][t.det_dn[k]]]
        ham = O.Real3IndexFactorization(O.COLLINEAR, M, nup, ndn, Likn[None], hij, 0.7, [Pu, Pd])
        for w in range(W):
            Tu, Td = Pu @ S_up[w], Pd @ S_dn[w]
            ov = np.linalg.det(Tu) * np.linalg.det(Td)
            G = np.concatenate([np.linalg.inv(Tu).T @ S_up[w].T, np.linalg.inv(Td).T @ S_dn[w].T])
            Ek = ham.energy(G[None])[0]
            num[w] += t.coef[k] * ov * Ek
            den[w] += t.coef[k] * ov
    ref = num / den[:, None]
    assert np.allclose(E, ref, rtol=1e-10, atol=1e-10), (E, ref)
    assert np.allclose(np.exp(logov), den, rtol=1e-10)


def test_phmsd_density_matrix_vs_single_determinants():
    """The Woodbury mixed density matrix against sum_k c_k ov_k G_k / sum_k c_k ov_k with G_k the
    full-space density matrix of determinant k, both mapped to the active orbitals:
    G_act[a][k] = sum over the trial's active rows, i.e. G_k^full = Phi_k (Phi_k^H S)^-1 ... ."""
    from safire_b200.synth import make_hamiltonian, make_phmsd_trial
    M, nup, ndn = 14, 4, 3
    h1, _ = make_hamiltonian(M, 2, 0.9, seed=5)
    _, C = np.linalg.eigh(h1)
    t = make_phmsd_trial(M, nup, ndn, C, nocc=3, nvirt=5, ndet=35, seed=5)
    rs = np.random.default_rng(9)
    W = 2
    S_up = (rs.standard_normal((W, M, nup)) + 1j * rs.standard_normal((W, M, nup))) / 4
    S_dn = (rs.standard_normal((W, M, ndn)) + 1j * rs.standard_normal((W, M, ndn))) / 4
    G, logov = P.phmsd_mixed_density_matrix(t, S_up, S_dn)
    # brute force: full density matrix of each determinant rho_k = S (D^H S)^-1 D^H, weighted
    occ = []
    for s in (0, 1):
        lst = [t.refc[s].copy()]
        for n in sorted(t.exc[s]):
            for e in t.exc[s][n]:
                o = t.refc[s].copy()
                o[e[:n]] = e[n:]
                lst.append(o)
        occ.append(lst)
    for w in range(W):
        num = [np.zeros((M, M), complex), np.zeros((M, M), complex)]
        den = 0j
        for k in range(t.coef.size):
            ov, rho = 1.0 + 0j, []
            for s, S in ((0, S_up[w]), (1, S_dn[w])):
                D = t.orbmat[s][occ[s][t.det_up[k] if s == 0 else t.det_dn[k]]]  # [N][M] = Phi^H
                T = D @ S
                ov *= np.linalg.det(T)
                rho.append(S @ np.linalg.inv(T) @ D)                        # [M][M]
            for s in (0, 1):
                num[s] += t.coef[k] * ov * rho[s]
            den += t.coef[k] * ov
        for s in (0, 1):
            full = (num[s] / den).T                                         # G[i][j] = <c_i^+ c_j>
            na = t.orbmat[s].shape[0]
            off = 0 if s == 0 else t.orbmat[0].shape[0]
            # compact (active-space) form: G_act = C_act^T-rotated rows, as the reference's
            # csrmm<'T'>(OrbMats, Gtmp) recovers the full one: full = OrbMats^T G_act
            Gact = G[w, off:off + na]
            assert np.allclose(t.orbmat[s].T @ Gact, full, atol=1e-10), s
        assert np.isclose(np.exp(logov[w]), den, rtol=1e-10)


def test_excitations_from_occupation_lists():
    """afqmc_phmsd_excitations (host code of the library, no GPU) turns occupation lists in
    arbitrary column order into the particle-hole structure: the Woodbury log overlap of the
    resulting trial equals the sum over the determinants as given, sum_k conj(c_k) det(D_k^H S)
    (the trial is sum_k c_k |D_k>; its couplings hold the conjugates)."""
    from safire_b200.synth import phmsd_trial_from_occupations
    rs = np.random.default_rng(9)
    M, nup, ndn, nact, ndet = 14, 4, 3, 10, 25
    A = np.linalg.qr(rs.standard_normal((M, M)) + 1j * rs.standard_normal((M, M)))[0]
    orb = [np.ascontiguousarray(A[:, :nact].conj().T)] * 2
    refc = [np.arange(nup), np.arange(ndn)]
    occ = []
    for nel in (nup, ndn):
        lst = [np.arange(nel)]
        while len(lst) < ndet:
            o = np.sort(rs.choice(nact, nel, replace=False))
            if rs.random() < 0.5:
                rs.shuffle(o)  # the coefficient refers to this column order
            lst.append(o)
        occ.append(np.array(lst))
    coef = rs.standard_normal(ndet) + 1j * rs.standard_normal(ndet)
    t = phmsd_trial_from_occupations(M, orb, refc, occ[0], occ[1], coef)
    W = 3
    Su = rs.standard_normal((W, M, nup)) + 1j * rs.standard_normal((W, M, nup))
    Sd = rs.standard_normal((W, M, ndn)) + 1j * rs.standard_normal((W, M, ndn))
    logov, _ = P.phmsd_log_overlap(t, Su, Sd)
    for w in range(W):
        tot = sum(np.conj(coef[k]) * np.linalg.det(orb[0][occ[0][k]] @ Su[w]) *
                  np.linalg.det(orb[1][occ[1][k]] @ Sd[w]) for k in range(ndet))
        assert abs(np.exp(logov[w]) - tot) <= 1e-10 * abs(tot)


@pytest.mark.parametrize("nex", [1, 2, 3, 4, 5])
def test_reduced_closed_form_matches_the_reference_sums(nex):
    """The reduced closed form the GPU tables kernels evaluate (phmsd.cu `excited_terms`,
    `excited_1body_all_kernel`), restated in numpy, against the reference's per-determinant
    sums (ph_excited_2body_energy_dense_cholesky / ph_excited_1body_energy over compact_R's
    rows).  With Q the inverse of the excitation block M[q][x] = QQ0[p_q][h_x]:
      Sf[j][c] = t_j[v_c] - sum_i t_j[r_i] QQ0[v_c][i],  SU[h][c] = sum_j t_h[r_j] Sf[j][c],
      P[a][b] = sum_q Sf[h_a][c_q] Q[b][q],  Kn = f0 + tr P,
      eX = sum_n (tr(P P) + 2 sum_{a,q} Q[a][q] SU[h_a][c_q]),
      e1 = sum_{p,q} Q[p][q] Sf1[h_p][c_q],  Sf1 = S[:, v] - S[:, r] QQ0[v, :]^T."""
    rs = np.random.default_rng(40 + nex)
    nw, nel, nchol, nact = 2, 6, 5, 13
    refc = np.arange(nel)
    virt = np.arange(nel, nact)

    def cx(*shape):
        return rs.standard_normal(shape) + 1j * rs.standard_normal(shape)

    T = cx(nw, nel, nchol, nact)
    S = cx(nw, nel, nact)
    QQ0 = cx(nw, nact, nel)
    for _ in range(3):
        holes = np.sort(rs.choice(nel, nex, replace=False))
        parts = np.sort(rs.choice(virt, nex, replace=False))
        iexcit = np.concatenate([holes, parts])[None]
        R = P.compact_R(iexcit, refc, QQ0)
        wgt = np.ones((1, nw), complex)
        EX, EJ, KE = P.ph_excited_2body_energy_dense_cholesky(iexcit, refc, T, R, wgt)
        E1 = P.ph_excited_1body_energy(iexcit, refc, S, R, wgt)
        cols = parts - nel  # particle columns among the virtual orbitals
        for w in range(nw):
            Q = np.linalg.inv(QQ0[w][np.ix_(parts, holes)])
            eX = 0j
            Kn = np.zeros(nchol, complex)
            for n in range(nchol):
                t = T[w, :, n, :]
                Sf = t[:, virt] - t[:, refc] @ QQ0[w][virt, :].T
                SU = t[:, refc] @ Sf
                Pm = Sf[np.ix_(holes, cols)] @ Q.T
                eX += np.trace(Pm @ Pm) + 2 * np.sum(Q * SU[np.ix_(holes, cols)])
                Kn[n] = sum(t[i, refc[i]] for i in range(nel)) + np.trace(Pm)
            assert abs(-0.5 * eX - EX[w]) <= 1e-10 * abs(EX[w])
            assert np.max(np.abs(Kn - KE[0, w])) <= 1e-10 * np.max(np.abs(KE[0, w]))
            Sf1 = S[w][:, virt] - S[w][:, refc] @ QQ0[w][virt, :].T
            e1 = np.sum(Q * Sf1[np.ix_(holes, cols)])
            assert abs(e1 - E1[w]) <= 1e-10 * abs(E1[w])
