"""Golden values of the reference's PHMSD component test, transcribed as constants, and the
deterministic fixture it evaluates them on.

Source: tests/test_phmsd_components.cpp of bkesk/SAFIRE (read as text).  The fixture (lines
33-96): ndet=50, nelec=5, nact=10, nchol=50, one walker, nex = 1..5 excitations per
determinant; Tna, R and wgt filled with sin/cos of their flat C-order index, the excitation
lists built by the probing loops below.  EXJ_REF[nex-1] = (EX, EJ) of
ph_excited_2body_energy_dense_cholesky (lines 41-47), checked with utils::Approx.
"""
import numpy as np

NDET, NELEC, NACT, NCHOL, NW = 50, 5, 10, 50, 1

EXJ_REF = np.array([
    [-3.710389910208285 - 666.8601775126258j, -448.4580805193352 + 260.52361637250124j],
    [257.47347099950423 + 1000.2224737398957j, -823.4796831379458 - 1004.1196065341555j],
    [782.6224431929506 - 1540.7376072631007j, -183.51974621436153 + 85.49030799002679j],
    [2023.4979464340804 - 36.30962737644677j, 1682.3242532758773 - 442.1588977259531j],
    [314.60033183810424 - 4993.354550714809j, -1238.764790338722 - 604.3447621988698j],
])


def fixture(nex):
    """(iexcit [ndet, 2*nex] int32, refc [nelec], Tna [nw,nelec,nchol,nact], R [nw,ndet,nex,nact],
    wgt [ndet,nw]) as test_phmsd_components.cpp:53-96 builds them."""
    i = np.arange(NW * NELEC * NCHOL * NACT)
    Tna = (np.sin(i) + 1j * np.cos(i * i)).reshape(NW, NELEC, NCHOL, NACT)
    i = np.arange(NW * NDET * nex * NACT)
    R = (np.sin(i * 3) + 1j * np.cos(i + i * i)).reshape(NW, NDET, nex, NACT)
    i = np.arange(NDET * NW)
    wgt = (np.sin(i * 2) + 1j * np.cos(i - 2 * i * i)).reshape(NDET, NW)
    iexcit = np.zeros((NDET, 2 * nex), dtype=np.int32)
    for nd in range(NDET):
        iocc = np.zeros(NELEC, dtype=np.int32)
        for k in range(nex):
            v = (k * k) % NELEC
            while iocc[v] != 0:
                v = (v + 1) % NELEC
            iocc[v] = 1
            iexcit[nd, k] = v
    for nd in range(NDET):
        iocc = np.zeros(NACT - NELEC, dtype=np.int32)
        for k in range(nex):
            v = (k + k * k) % (NACT - NELEC)
            while iocc[v] != 0:
                v = (v + 1) % (NACT - NELEC)
            iocc[v] = 1
            iexcit[nd, k + nex] = v + NELEC
    refc = np.arange(NELEC, dtype=np.int32)
    return iexcit, refc, Tna, R, wgt
