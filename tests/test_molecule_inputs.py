"""Molecular inputs on the CPU: the HDF5 reader against the committed fixtures, the PHMSD trial
built from the reference's files against a brute-force sum over its explicit determinants
(overlaps and local energies, with complex orbitals and coefficients), the several-determinant
trial density, and the JSON input parser."""
import importlib.util
import os

import numpy as np
import pytest

from oracle import afqmc as O
from oracle import phmsd as OP
from safire_b200 import inputs as I
from safire_b200 import molecule as Mo
from tests import molecule_fixtures as F

HERE = os.path.dirname(os.path.abspath(__file__))


def _fixture_script():
    spec = importlib.util.spec_from_file_location(
        "make_molecule_fixtures", os.path.join(HERE, "golden", "make_molecule_fixtures.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_reader_reproduces_fixtures():
    """The committed arrays are what safire_b200.h5 reads from the reference's files (checked
    where the reference checkout is present)."""
    mk = _fixture_script()
    if not os.path.isdir(mk.INP):
        pytest.skip("reference inputs not present")
    for key, rel in mk.HAMS.items():
        h = I.read_hamiltonian(os.path.join(mk.INP, rel))
        ref = F.hamiltonian(key)
        assert np.array_equal(h.hcore, ref.hcore) and np.array_equal(h.Likn, ref.Likn)
        assert h.nuclear_energy == ref.nuclear_energy
    for key, rel in mk.WFNS.items():
        w = I.read_wavefunction(os.path.join(mk.INP, rel))
        ref = F.wavefunction(key)
        assert type(w) is type(ref) and w.walker_type == ref.walker_type
        assert np.array_equal(w.ci, ref.ci)
        if isinstance(w, I.NOMSDInput):
            for a, b in zip(w.PsiT, ref.PsiT):
                assert all(np.array_equal(x, y) for x, y in zip(a, b))
        else:
            assert np.array_equal(w.occa, ref.occa) and np.array_equal(w.occb, ref.occb)
            assert all(np.array_equal(x, y) for x, y in zip(w.references, ref.references))


def test_fixture_contents():
    """Shapes and the settings of the statistical references."""
    h = F.hamiltonian("bh")
    assert h.hcore.shape == (1, 19, 19) and h.Likn.shape == (1, 19, 19, 78)
    assert abs(h.energy_offset(I.CLOSED, 3, 3) - 1.428972809786131) < 1e-15
    w = F.wavefunction("bh_rhf_nomsd")
    assert (w.walker_type, w.M, w.nup, w.ndn, w.ci.size) == (I.CLOSED, 19, 3, 3, 1)
    assert np.allclose(w.PsiT[0][0] @ w.PsiT[0][0].conj().T, np.eye(3))
    refs = F.references()
    assert len(refs) == 12
    for r in refs.values():
        assert r["walkers"] == 1536 and r["timestep"] == 0.01 and r["energy_error"] > 0


def _expanded(w):
    orb = [w.references[0], w.references[-1]] if w.references else [np.eye(w.M)] * 2
    return [[orb[0][oa], orb[1][ob]] for oa, ob in zip(w.occa, w.occb)]


def _walkers(M, nup, ndn, W, seed):
    rs = np.random.default_rng(seed)
    Su = rs.standard_normal((W, M, nup)) + 1j * rs.standard_normal((W, M, nup))
    Sd = rs.standard_normal((W, M, ndn)) + 1j * rs.standard_normal((W, M, ndn))
    return Su, Sd


@pytest.mark.parametrize("key", ["bh_casci_rhf_phmsd", "bh_casci_uhf_phmsd", "n2_cas_phmsd"])
def test_phmsd_overlap_vs_explicit_determinants(key):
    """<Psi_T|phi> = sum_k conj(c_k) det(D_k^H phi_up) det(D_k^H phi_dn) over the file's
    determinants in their own orbital order: the particle-hole structure, the permutation
    signs and the conjugated couplings of phmsd_trial reproduce it."""
    w = F.wavefunction(key)
    tr = I.phmsd_trial(w)
    Su, Sd = _walkers(w.M, w.nup, w.ndn, 3, 0)
    lo, _ = OP.phmsd_log_overlap(tr, Su, Sd)
    bf = sum(np.conj(c) * np.linalg.det(D[0] @ Su) * np.linalg.det(D[1] @ Sd)
             for c, D in zip(w.ci, _expanded(w)))
    assert np.max(np.abs(np.exp(lo) - bf)) < 1e-12 * np.max(np.abs(bf))


def test_phmsd_energy_vs_explicit_determinants():
    """The Woodbury local energy of the rotated complex CASCI trial equals the
    several-determinant NOMSD local energy over the same determinants written out."""
    w = F.wavefunction("bh_casci_rhf_phmsd")
    h = F.hamiltonian("bh")
    tr = I.phmsd_trial(w)
    E0 = h.energy_offset(I.COLLINEAR, w.nup, w.ndn)
    hij = np.concatenate([h.hcore, h.hcore])
    Su, Sd = _walkers(w.M, w.nup, w.ndn, 2, 1)
    E, lo = OP.phmsd_energy(tr, OP.ActiveSpaceHamiltonian(tr, h.Likn, hij, E0), Su, Sd)
    dets = _expanded(w)
    hams = [O.Real3IndexFactorization(I.COLLINEAR, w.M, w.nup, w.ndn, h.Likn, hij, E0, D)
            for D in dets]
    md = O.NOMSDMulti(hams, dets, w.ci)
    Em, lom = md.Energy(Su, Sd)
    assert np.max(np.abs(E - Em)) < 1e-9 * np.max(np.abs(Em))
    assert np.max(np.abs(np.exp(lo) - np.exp(lom))) < 1e-10 * np.max(np.abs(np.exp(lom)))


def test_several_determinant_trial_density():
    """Trace N per spin; a single determinant gives its projector; the CASCI expansion keeps
    only the non-orthogonal pairs (the 529 exactly orthogonal ones add nothing)."""
    w1 = F.wavefunction("bh_rhf_nomsd")
    g1 = Mo.nomsd_mean_field_density(w1.PsiT, w1.ci, w1.walker_type)
    P = w1.PsiT[0][0]
    assert np.allclose(g1[0], P.T @ P.conj())
    w = F.wavefunction("bh_casci_rhf_nomsd")
    g = Mo.nomsd_mean_field_density(w.PsiT, w.ci, w.walker_type)
    assert abs(np.trace(g[0]) - w.nup) < 1e-12
    # brute force over pairs p <= q with a non-singular T
    num = np.zeros((w.M, w.M), complex)
    den = 0.0
    for p in range(w.ci.size):
        for q in range(p, w.ci.size):
            A, B = w.PsiT[q][0], w.PsiT[p][0].conj().T
            T = A @ B
            if abs(np.linalg.det(T)) < 1e-12:
                continue
            s = (np.conj(w.ci[q]) * w.ci[p] * np.linalg.det(T)).real
            num += s * (A.T @ np.linalg.inv(T).T @ B.T)
            den += s
    assert np.allclose(g[0], num / den, atol=1e-13)
    wu = F.wavefunction("bh_uhf_nomsd")
    gu = Mo.nomsd_mean_field_density(wu.PsiT, wu.ci, wu.walker_type)
    assert gu.shape == (2, 19, 19)
    assert abs(np.trace(gu[0]) - 3) < 1e-12 and abs(np.trace(gu[1]) - 3) < 1e-12


def test_json_input_parser():
    doc = {"seed": 42, "execute": {
        "walker_set": {"walker_type": "CLOSED"}, "wavefunction": {"filename": "w.h5"},
        "hamiltonian": {"filename": "h.h5"}, "timestep": 0.01, "steps": 12000,
        "n_walkers_per_mpi_task": 16, "population_control_interval": 10,
        "measure_interval": 10, "walker_ortho_interval": 10, "equilibration_steps": 3000}}
    c = Mo.parse_input(doc)
    assert (c["walkers"], c["steps"], c["walker_type"]) == (16, 12000, I.CLOSED)
    assert (c["rp"].walker_ortho_interval, c["rp"].equilibration_steps, c["rp"].seed) == \
        (10, 3000, 42)
    doc["execute"]["walker_set"]["walker_type"] = "NONCOLLINEAR"
    with pytest.raises(ValueError):
        Mo.parse_input(doc)
    del doc["execute"]["walker_set"]
    del doc["execute"]["n_walkers_per_mpi_task"]
    with pytest.raises(ValueError):
        Mo.parse_input(doc)


def test_blocked_mean():
    rs = np.random.default_rng(3)
    x = rs.standard_normal(1600)
    m, e = Mo.blocked_mean(x)
    assert abs(m - x.mean()) < 1e-15
    assert 0.5 / 40 < e < 2.0 / 40  # ~ 1 / sqrt(1600) for independent samples


def _random_orbitals(rs, M, complex_=True):
    A = rs.standard_normal((M, M)) + (1j * rs.standard_normal((M, M)) if complex_ else 0)
    Q = np.linalg.qr(A)[0]
    return np.ascontiguousarray(Q.conj().T)  # rows: conjugated orbitals


def test_phmsd_mean_field_single_determinant_is_nomsd():
    """One determinant: the PHMSD mean field equals NOMSD::vMF of that determinant."""
    from safire_b200.synth import phmsd_trial_from_occupations
    rs = np.random.default_rng(4)
    M, nup, ndn, Nc, dt = 9, 3, 2, 7, 0.01
    orb = _random_orbitals(rs, M)
    L = rs.standard_normal((1, M, M, Nc))
    L = 0.5 * (L + L.transpose(0, 2, 1, 3))
    refc = [np.arange(nup), np.arange(ndn)]
    tr = phmsd_trial_from_occupations(M, [orb, orb], refc, refc[0][None], refc[1][None],
                                      np.array([0.7 - 0.2j]))
    v = Mo.phmsd_mean_field(tr, L, dt)
    psi = [orb[:nup], orb[:ndn]]
    hij = np.zeros((2, M, M), complex)
    ham = O.Real3IndexFactorization(I.COLLINEAR, M, nup, ndn, L, hij, 0.0, psi)
    assert np.allclose(v, O.NOMSD(ham, psi).vMF(dt), atol=1e-13)


def test_phmsd_mean_field_single_excitation_is_exact():
    """Two determinants one alpha excitation apart (0 1 -> 0 2, sign +1) with real orbitals: the
    restated mean field equals the force bias of the exact one-body density of the expansion."""
    from safire_b200.synth import phmsd_trial_from_occupations
    rs = np.random.default_rng(5)
    M, Nc, dt = 8, 6, 0.02
    orb = _random_orbitals(rs, M, complex_=False).astype(np.complex128)
    L = rs.standard_normal((1, M, M, Nc))
    L = 0.5 * (L + L.transpose(0, 2, 1, 3))
    occa = np.array([[0, 1], [0, 2]])
    occb = np.array([[0, 1], [0, 1]])
    c = np.array([0.9, -0.4])
    tr = phmsd_trial_from_occupations(M, [orb, orb], [occa[0], occb[0]], occa, occb, c)
    v = Mo.phmsd_mean_field(tr, L, dt)
    norm = np.sum(c ** 2)
    ga = np.zeros((M, M))
    ga[[0, 1], [0, 1]] += c[0] ** 2 / norm
    ga[[0, 2], [0, 2]] += c[1] ** 2 / norm
    ga[1, 2] = ga[2, 1] = c[0] * c[1] / norm
    gb = np.zeros((M, M))
    gb[[0, 1], [0, 1]] = 1.0
    R = orb.real
    exact = sum(np.einsum("ik,ikn->n", R.T @ g @ R, L[0]) for g in (ga, gb)) * np.sqrt(dt)
    assert np.allclose(v, exact, atol=1e-13)


def test_h5_reader_rejects_other_files(tmp_path):
    from safire_b200.h5 import File
    p = tmp_path / "not.h5"
    p.write_bytes(b"\x00" * 600 + b"\x89HDF\r\n\x1a\n" + b"\x00" * 100)  # signature off-grid
    with pytest.raises(ValueError):
        File(str(p))
    p.write_bytes(b"plain text, no superblock")
    with pytest.raises(ValueError):
        File(str(p))
