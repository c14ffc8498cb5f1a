"""Pins the oracle (CPU restatement) before anything is checked against it."""
import os
import subprocess

import numpy as np
import pytest

from oracle import afqmc as O
from tests.golden import sdet_ops_golden as g

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _B():
    return np.repeat(g.M_B[None], g.NWALK, 0).copy()


def test_log_overlap_golden():
    ov = np.zeros(g.NWALK, complex)
    O.Log_Overlap(g.M_A, _B(), ov)
    assert g.approx(ov, np.full(g.NWALK, g.OV_BASE))
    ov = np.zeros(g.NWALK, complex)
    O.Log_Overlap(g.M_A[:2, :3], _B()[:, :3, :2].copy(), ov)
    assert g.approx(ov, np.full(g.NWALK, g.OV2_BASE))


@pytest.mark.parametrize("compact", [False, True])
def test_mixed_density_matrix_golden(compact):
    ov = np.zeros(g.NWALK, complex)
    G = O.MixedDensityMatrix(g.M_A, _B(), ov, compact=compact)
    ref = g.VC_REF if compact else g.V_REF
    assert g.approx(G, np.repeat(ref[None], g.NWALK, 0))
    assert g.approx(ov, np.full(g.NWALK, g.OV_BASE))
    ov = np.zeros(g.NWALK, complex)
    G = O.MixedDensityMatrix(g.M_A[:2, :3], _B()[:, :3, :2].copy(), ov, compact=compact)
    ref = g.VC_REF_2 if compact else g.V_REF_2
    assert g.approx(G, np.repeat(ref[None], g.NWALK, 0))


def test_inverse_logdet_golden():
    ld = np.zeros(g.NWALK, complex)
    inv = O.inverse_logdet(np.repeat(g.INV_A[None], g.NWALK, 0), ld)
    assert g.approx(inv, np.repeat(g.INV_REF[None], g.NWALK, 0))
    assert g.approx(ld, np.full(g.NWALK, g.LOGDET_INV_REF))


def test_orthogonalize_golden():
    # test_sdet_ops.cpp:296-304: after orthogonalize, Log_Overlap(Q, Q) == 0
    Q = _B()
    ld = np.zeros(g.NWALK, complex)
    O.orthogonalize(Q, ld)
    ov = np.array([np.log(np.linalg.det(Q[w].conj().T @ Q[w])) for w in range(g.NWALK)])
    assert g.approx(ov, np.zeros(g.NWALK))
    # R has a positive real diagonal: Q^H B is upper triangular with positive diagonal
    R = Q[0].conj().T @ g.M_B
    assert np.all(np.diag(R).real > 0)
    assert np.allclose(np.tril(R, -1), 0, atol=1e-12)


def test_rng_matches_libstdcxx():
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "all", "check_ref"])
    seed = O.split_seed(0, 0, 1)
    rng = O.HostRandomGenerator(seed)
    ours = rng.sample_uniform(5000)
    out = subprocess.check_output([os.path.join(ROOT, "oracle", "_ref", "stdrng_ref"), str(seed),
                                   "5000"])
    ref = np.array([float(x) for x in out.split()])
    assert np.array_equal(ours, ref)


def test_split_seed_known_values():
    # splitmix64 finalizer of (seed<<32 | stream<<24 | rank) + golden ratio increment
    x = (0 << 32 | 1 << 24 | 0) + 0x9E3779B97F4A7C15
    x &= (1 << 64) - 1
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & ((1 << 64) - 1)
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & ((1 << 64) - 1)
    x ^= x >> 31
    assert O.split_seed(0, 0, 1) == x


def test_comb_preserves_population():
    rng = O.HostRandomGenerator(O.split_seed(3, 0, 0))
    w = np.random.default_rng(1).random(200) * 2
    w[5] = 0.0
    off = O.comb(rng, w, 200)
    assert off.sum() == 200
    assert off[5] == 0
    # expected copies follow the weights
    exp = w / w.sum() * 200
    assert np.all(np.abs(off - exp) <= 1.0 + 1e-12)


def test_comb_collapse_raises():
    rng = O.HostRandomGenerator(1)
    with pytest.raises(RuntimeError):
        O.comb(rng, np.zeros(8), 8)


def test_plan_walker_exchange_invariants():
    rs = np.random.default_rng(7)
    for _ in range(50):
        nr = rs.integers(1, 6)
        counts = list(rs.integers(1, 9, size=nr))
        ntot = sum(counts)
        off = np.zeros(ntot, dtype=int)
        for _k in range(ntot):
            off[rs.integers(0, ntot)] += 1
        plan = O.plan_walker_exchange(off, counts)
        # after the plan every rank holds counts[r] walkers
        held = []
        first = 0
        for r, nw in enumerate(counts):
            held.append(int(off[first:first + nw].sum()))
            first += nw
        for src, wk, dst, n in plan:
            held[src] -= n
            held[dst] += n
            assert src != dst and n > 0
        assert held == counts


def test_probit_symmetry_and_regions():
    p = np.array([1e-6, 0.01, 0.02425, 0.3, 0.5, 0.7, 0.97575, 0.99, 1 - 1e-6])
    x = O.probit(p)
    assert np.allclose(x, -O.probit(1 - p), atol=1e-9)
    assert x[4] == 0.0
    assert O.probit(np.array([0.0]))[0] == -np.inf


def test_oracle_step_sanity():
    from safire_b200.synth import make_workload
    wl = make_workload("cfg1", W=8)
    ham = O.Real3IndexFactorization(wl.walker_type, wl.M, wl.nup, wl.ndn, wl.Likn, wl.hij, wl.E0,
                                    wl.PsiT)
    wfn = O.NOMSD(ham, wl.PsiT)
    # trial density matrix is idempotent with trace N (test_wfn_factory.cpp:206-218)
    SA, _ = wfn.initial_walker()
    ov = np.zeros(1, complex)
    Gf = O.MixedDensityMatrix(wl.PsiT[0], SA[None], ov, compact=False)[0]
    assert abs(np.trace(Gf) - wl.nup) < 1e-12
    assert np.allclose(Gf @ Gf, Gf, atol=1e-12)
    prop = O.Propagator(wfn, O.PropagatorParams(dt=wl.dt))
    ws = O.WalkerSet.from_trial(wfn, 8)
    en, _ = O.run_afqmc(wfn, prop, ws, O.RunParams(steps=12, equilibration_steps=5))
    assert np.all(np.isfinite(ws.props))
    assert len(en) == 1 and np.isfinite(en[0][1])


def test_exchange_energy_independent_loop():
    """EXX of the oracle against an independent O(N^2 M^2 Nc) loop over the Cholesky vectors."""
    from safire_b200.synth import make_workload
    wl = make_workload("cfg1", W=2, M=8, N=3, Nc=6)
    ham = O.Real3IndexFactorization(wl.walker_type, wl.M, wl.nup, wl.ndn, wl.Likn, wl.hij, wl.E0,
                                    wl.PsiT)
    rs = np.random.default_rng(0)
    G = rs.standard_normal((2, 3 * 8)) + 1j * rs.standard_normal((2, 3 * 8))
    E = ham.energy(G)
    L = wl.Likn[0]
    P = wl.PsiT[0]
    for w in range(2):
        Gw = G[w].reshape(3, 8)
        ex = 0j
        kl = np.zeros(6, complex)
        for n in range(6):
            Ln = P @ L[:, :, n]  # Lnak[n]
            T = Gw @ Ln.T        # T[b, a]
            ex += np.sum(T * T.T)
            kl[n] = np.trace(T)
        assert abs(E[w, 1] - (-0.5 * 2 * ex)) < 1e-12 * max(1, abs(ex))
        assert abs(E[w, 2] - 0.5 * 4 * np.sum(kl * kl)) < 1e-12 * max(1, abs(E[w, 2]))
