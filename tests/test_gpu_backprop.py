"""Back-propagated one-body density matrix on the GPU (safire_b200.backprop): the estimate
against the oracle's restatement from the same recorded fields, factors, anchors and weights
(CLOSED and COLLINEAR, with combs and re-orthogonalisations inside the window); the recorded
fields against construct_X of the step's force bias and uniforms; the path-restoration factors
against the step's bounded local energy; and the BH RHF back-propagated density matrix against
the reference's statistical result."""
import math

import numpy as np
import pytest
import torch

from oracle import afqmc as O
from oracle import backprop as OB
from safire_b200 import afqmc as A
from safire_b200 import capi
from safire_b200.backprop import BackPropagation
from safire_b200.driver import RunParams, Simulation
from safire_b200.synth import make_workload
from tests import molecule_fixtures as F

pytestmark = pytest.mark.gpu


class _Checked(BackPropagation):
    """Compares every estimate with the oracle's from the same state."""

    def __init__(self, *a, oham=None, **k):
        super().__init__(*a, **k)
        self.oham = oham
        self.checked = 0

    def estimate(self, nbp):
        sim = self.sim
        slots = [(self.pos - nbp + j) % self.nback for j in range(nbp)]  # oldest first
        V_hist = [self.oham.vHS(self.X[s].cpu().numpy(), sim.dt) for s in slots]
        P1, _ = sim.prop.P1_vMF()
        refs = [np.repeat(t.cpu().numpy()[0][None], self.W, axis=0) for t in self.trial]
        OB.back_propagate(refs, list(P1), V_hist, self.order, self.ortho)
        w0 = sim.wset.properties()[:, capi.WEIGHT].cpu().numpy()
        w = OB.path_restored_weights(w0, self.F[slots].cpu().numpy())
        ref = OB.bp_onerdm(refs, [a.cpu().numpy() for a in self.anchor], w)
        out = super().estimate(nbp)
        got = out.cpu().numpy()
        assert np.max(np.abs(got - ref)) < 1e-9 * max(1.0, np.max(np.abs(ref))), \
            np.max(np.abs(got - ref))
        self.checked += 1
        return out


def _run_checked(wl, W, steps, nback, ortho):
    rp = RunParams(walker_ortho_interval=4, population_control_interval=3, measure_interval=2,
                   equilibration_steps=2, seed=3)
    sim = Simulation.from_workload(wl, W=W, rp=rp)
    oham = O.Real3IndexFactorization(wl.walker_type, wl.M, wl.nup, wl.ndn, wl.Likn, wl.hij,
                                     wl.E0, wl.PsiT)
    bp = _Checked(sim, wl.PsiT, steps=nback, ortho_interval=ortho, oham=oham)
    for _ in range(steps):
        sim.step()
    torch.cuda.synchronize()
    return sim, bp


def test_backprop_closed_vs_oracle(cuda):
    wl = make_workload("cfg1", W=12)
    sim, bp = _run_checked(wl, 12, 2 + 3 * 5, nback=5, ortho=2)
    assert bp.checked == 3 and len(bp.samples) == 3
    g = bp.samples[-1][1][0]
    assert abs(np.trace(g) - wl.nup) < 1e-9


def test_backprop_collinear_vs_oracle(cuda):
    from safire_b200 import molecule as Mo
    ham, wfn, wt, _ = F.case("bh_uhf_collinear")
    wl, _ = Mo._workload(ham, wfn, 16, 0.01, wt)
    sim, bp = _run_checked(wl, 16, 2 + 2 * 7, nback=7, ortho=3)
    assert bp.checked == 2
    g = bp.samples[-1][1]
    assert abs(np.trace(g[0]) - wl.nup) < 1e-9 and abs(np.trace(g[1]) - wl.ndn) < 1e-9


def test_recorded_fields_and_factors(cuda):
    """X of the step = construct_X(vbias, u, vMF) (the force-bias fields the step used); the
    factor = exp(-i dt Im eloc) / max(0, cos dtheta) with the step's bounded local energy."""
    wl = make_workload("cfg1", W=8)
    rp = RunParams(walker_ortho_interval=100, population_control_interval=100,
                   measure_interval=100, equilibration_steps=0, seed=5)
    sim = Simulation.from_workload(wl, W=8, rp=rp)
    bp = BackPropagation(sim, wl.PsiT, steps=4)
    rs = np.random.default_rng(2)
    _, vMF = sim.prop.P1_vMF()
    vMF = vMF.real.astype(np.complex128)
    for _ in range(3):
        u = rs.random((8, wl.Nc))
        sim.step(uniforms=torch.as_tensor(u, device="cuda"), measure=False)
        torch.cuda.synchronize()
        last = sim.prop.last_step(8)
        X_ref, _ = O.construct_X(last.vbias.cpu().numpy(), u, vMF, sim.prop.params.vbias_bound)
        X_rec = bp.X[(bp.pos - 1) % bp.nback].cpu().numpy()
        assert np.max(np.abs(X_rec - X_ref)) < 1e-10 * np.max(np.abs(X_ref))
        p = sim.wset.properties().cpu().numpy()
        scale = np.maximum(0.0, np.cos(p[:, capi.THETA].real))
        ph = np.exp(-1j * sim.dt * p[:, capi.PSEUDO_ELOC].imag)
        want = np.where(scale > 0, ph / np.where(scale > 0, scale, 1.0), 0.0)
        got = bp.F[(bp.pos - 1) % bp.nback].cpu().numpy()
        assert np.max(np.abs(got - want)) < 1e-12


def test_bh_rhf_backpropagated_onerdm_vs_reference(cuda):
    """The reference's BackPropEstimator/Steps=100/OneRDM of BH (RHF trial, CLOSED, 1536
    walkers, path restoration): every element within five combined standard errors."""
    from safire_b200 import molecule as Mo
    ham, wfn, wt, r = F.case("bh_rhf_closed")
    rp = RunParams(walker_ortho_interval=r["walker_ortho_interval"],
                   population_control_interval=r["population_control_interval"],
                   measure_interval=r["measure_interval"], equilibration_steps=3000,
                   seed=r["seed"])
    sim = Mo.simulation(ham, wfn, r["walkers"], r["timestep"], wt, rp)
    bp = BackPropagation(sim, [wfn.PsiT[0][0]], steps=r["bp_steps"],
                         ortho_interval=r["walker_ortho_interval"],
                         path_restoration=r["bp_path_restoration"])
    for _ in range(3000 + 9600):
        sim.step()
    torch.cuda.synchronize()
    g = np.array([s[1][0] for s in bp.samples]).real     # [samples][M][M]
    assert len(g) >= 90
    nb = 16
    n = g.shape[0] // nb
    blocks = g[g.shape[0] - nb * n:].reshape(nb, n, *g.shape[1:]).mean(1)
    mean, err = g.mean(0), blocks.std(0, ddof=1) / math.sqrt(nb)
    ref = np.array(r["bp_onerdm_real"])[0]
    ref_err = np.array(r["bp_onerdm_error_real"])[0]
    assert abs(np.trace(mean) - 3.0) < 1e-8
    z = np.abs(mean - ref) / np.sqrt(err ** 2 + ref_err ** 2 + 1e-14)
    assert np.max(z) < 5.0, (np.unravel_index(np.argmax(z), z.shape), np.max(z))
