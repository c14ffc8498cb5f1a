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
