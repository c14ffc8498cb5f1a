"""Back-propagated one-body density matrix (Estimators/BackPropEstimator.hpp,
Propagators/AFQMCBasePropagator.cpp:403-533).

`BackPropagation` attaches to a safire_b200.driver.Simulation as an observer and keeps, as the
reference's walker set does (WalkerSetBase.h:493-530, WalkerSetUpdate.hpp:128-187):
- the auxiliary fields X [nback][W][Nc] of every step, read from the step's own field buffer;
- the per-step path-restoration factor of every walker, w / |w| / max(0, cos dtheta) (zero where
  the projection or a non-finite energy killed it), formed from the phase and the dtheta the
  update kernel writes: the new phase over the old one is w / |w|;
- the walkers at the start of the window (the anchor, SlaterMatrixN).
The comb copies walkers into the slots of the ones it removes; the histories and anchors follow
with the same slot map (a walker keeps its slot, extra copies fill the emptied slots in
increasing order, as afqmc_population_control does).

At the end of each window of `steps` steps (BackPropEstimator::measure) the trial, one copy per
walker, is propagated backwards through the stored fields, newest first:
S <- P1^H sum_n (-i V^H)^n / n! P1^H S with V = vHS(X) (the library's afqmc_propagate given P1^H
and -V^H), re-orthogonalised with afqmc_orthogonalize every `ortho_interval` steps and at the
end.  The estimate is sum_w w'_w G_w / sum_w w'_w, w' the weights times the factors of the
window, G_w = (B T^-1 A^H)^T with A the back-propagated trial, B the anchor and T = A^H B
(afqmc_mixed_density_matrix_batched: DMMA products and the library's Gauss-Jordan inverse, the
reference's batched-bra det_ops::MixedDensityMatrix).  Then the window
restarts from the current walkers.  A trial of several determinants back-propagates each of its
references (NOMSD: its determinants; PHMSD: its configurations, phmsd_references) and weights
their density matrices by their shares of each walker's overlap.  One walker set on one GPU.
"""
from __future__ import annotations

import numpy as np
import torch

from . import afqmc as A
from . import capi
from .capi import COLLINEAR


def slot_map(offspring):
    """Source walker of every slot after the single-rank comb: a walker with offspring >= 1
    keeps its slot, its extra copies fill the slots of the walkers without offspring in
    increasing order (population_control.hpp:142-209)."""
    off = np.asarray(offspring)
    src = np.arange(off.size)
    free = np.nonzero(off == 0)[0]
    nxt = 0
    for i in range(off.size):
        for _ in range(1, int(off[i])):
            src[free[nxt]] = i
            nxt += 1
    if nxt != free.size:
        raise ValueError("offspring counts do not conserve the population")
    return src


def phmsd_references(trial):
    """The references of a PHMSD trial for back propagation (PHMSD.hpp:232-279): one per
    determinant, its configuration's orbitals in excitation order (the rows of orbmat it
    occupies, per spin [N_s][M]), weighted by its coefficient with the permutation sign, c_k =
    conj(coupling k)."""
    refs = []
    confs = []
    for s in (0, 1):
        ref = np.asarray(trial.refc[s])
        cs = [ref.copy()]
        for n in sorted(trial.exc[s]):
            for e in trial.exc[s][n]:
                c = ref.copy()
                c[e[:n]] = e[n:]
                cs.append(c)
        confs.append(cs)
    for k in range(len(trial.coef)):
        psi = [np.asarray(trial.orbmat[s])[confs[s][int((trial.det_up, trial.det_dn)[s][k])]]
               for s in (0, 1)]
        refs.append((complex(np.conj(trial.coef[k])), psi))
    return refs


def reference_onerdm(refs, walkers, weights, ref_w, log_offset, closed_factor):
    """sum_w weights_w sum_d share_{w,d} G_{w,d} / sum_w weights_w per spin [nspin][M][M]: the
    reference loop of BackPropEstimator.hpp:36-120 / MixedEstimator.hpp:40-105 with onerdm.hpp.
    refs: per spin the references, one copy per walker, [nref * W][M][N_s] (reference-major);
    walkers: per spin [W][M][N_s]; log_offset [nref][W] added to the log overlaps (the BP
    log det shift, or minus the walkers' OVLP); closed_factor multiplies the one block's log
    overlap of CLOSED walkers (2 in back propagation, 1 in the mixed estimator).  The log overlap
    of reference d with walker w is log det(A^H B) over the spins, its
    overlap conj(c_d) e^{log}, its share that over the walker's sum, G_{w,d} = (B T^-1 A^H)^T."""
    nr = len(ref_w)
    W, M = walkers[0].shape[0], walkers[0].shape[1]
    dev = walkers[0].device
    lo = log_offset.clone()
    Gs = []
    for Aref, B in zip(refs, walkers):
        N = B.shape[2]
        if N == 0:
            Gs.append(None)
            continue
        Bd = B.unsqueeze(0).expand(nr, -1, -1, -1).reshape(nr * W, M, N).contiguous()
        G = torch.empty((nr * W, M, M), dtype=torch.complex128, device=dev)
        ld = torch.zeros(nr * W, dtype=torch.complex128, device=dev)
        A.det_ops.MixedDensityMatrixBatched(Aref.contiguous(), Bd, G, ld, compact=False)
        lo = lo + closed_factor * ld.view(nr, W)
        Gs.append(G.view(nr, W, M, M))
    cw = torch.as_tensor(np.conj(np.asarray(ref_w, dtype=np.complex128)), device=dev)[:, None]
    # shares ov_d / sum_d ov_d with ov_d = conj(c_d) e^{lo_d}: a common factor per walker
    # cancels, so the largest real part comes off before the exponential
    lo = lo - lo.real.max(0, keepdim=True).values
    ov = cw * torch.exp(lo)
    share = ov / ov.sum(0, keepdim=True)
    out = []
    for G in Gs:
        if G is None:
            out.append(torch.zeros((M, M), dtype=torch.complex128, device=dev))
            continue
        out.append(torch.einsum("w,dw,dwik->ik", weights, share, G) / weights.sum())
    return torch.stack(out)


def mixed_onerdm(sim, references):
    """The mixed estimator's one-body density matrix of the current walkers
    (MixedEstimator.hpp:40-105, onerdm.hpp) over the trial's references [(c_d, per-spin
    PsiT_d)]: reference_onerdm with the references unpropagated, the walkers' stored log
    overlaps subtracted, and no doubling for CLOSED walkers (the reference loops over the spin
    blocks it has).  Returns [nspin][M][M] (device)."""
    ham = sim.ham
    nsp = 2 if ham.walker_type == COLLINEAR else 1
    W, M = sim.wset.W, ham.M
    dev = sim.wset.buffer.device
    nr = len(references)
    refs = []
    for s in range(nsp):
        R = torch.as_tensor(np.ascontiguousarray(np.stack(
            [np.asarray(P[s]).conj().T for _, P in references])), device=dev)
        refs.append(R.unsqueeze(1).expand(-1, W, -1, -1).reshape(nr * W, M, R.shape[2])
                    .contiguous())
    walkers = [sim.wset.SlaterMatrices(s).contiguous() for s in range(nsp)]
    props = sim.wset.properties()
    shift = -props[:, capi.OVLP].unsqueeze(0).expand(nr, -1)
    return reference_onerdm(refs, walkers, props[:, capi.WEIGHT].clone(),
                            [c for c, _ in references], shift, 1.0)


class BackPropagation:
    def __init__(self, sim, PsiT=None, steps=100, ortho_interval=None, path_restoration=True,
                 references=None):
        """sim: a Simulation; PsiT: its single-determinant trial, per spin [N_s][M] (host); or
        references: the trial's determinants [(c_d, per-spin PsiT_d)] as the reference's
        getReferences / getReferenceWeight give them (NOMSD: its determinants and ci;
        PHMSD: phmsd_references)."""
        ham = sim.ham
        if references is None:
            if PsiT is None:
                raise ValueError("give the trial's PsiT or its references")
            references = [(1.0 + 0j, PsiT)]
        if steps <= 0:
            raise ValueError("steps must be positive")
        self.sim = sim
        self.nback = int(steps)
        self.ortho = int(ortho_interval or sim.rp.walker_ortho_interval)
        self.path_restoration = path_restoration
        self.collinear = ham.walker_type == COLLINEAR
        self.nel = [ham.nup] + ([ham.ndn] if self.collinear else [])
        W, M, Nc = sim.wset.W, ham.M, ham.Nc
        dev = sim.wset.buffer.device
        self.W, self.M, self.dev = W, M, dev
        self.X = torch.zeros((self.nback, W, Nc), dtype=torch.complex128, device=dev)
        self.F = torch.ones((self.nback, W), dtype=torch.complex128, device=dev)
        self.pos = 0
        P1, _ = sim.prop.P1_vMF()
        self.P1h = [torch.as_tensor(np.ascontiguousarray(P1[s].conj().T), device=dev)
                    for s in range(P1.shape[0])]
        nsp = len(self.nel)
        self.ref_w = np.array([complex(c) for c, _ in references])
        # per spin, the references' Slater matrices PsiT_d^H stacked [nref][M][N_s]
        self.trial = [torch.as_tensor(np.ascontiguousarray(np.stack(
            [np.asarray(P[s]).conj().T for _, P in references])), device=dev)
            for s in range(nsp)]
        self.nref = len(references)
        self.order = int(getattr(sim.prop.params, "taylor_n", 6))
        self.samples = []  # (step, [nspin][M][M] on the host)
        self._phase0 = None
        self._set_anchor(sim.step_index - 1)
        sim.observers.append(self)

    # ---------------------------------------------------------------- walker data
    def _slater(self, s):
        return self.sim.wset.SlaterMatrices(s)

    def _set_anchor(self, step):
        self.anchor = [self._slater(s).clone() for s in range(len(self.nel))]
        self.bp_pos = step

    # ---------------------------------------------------------------- observer hooks
    def before_step(self, sim):
        self._phase0 = sim.wset.properties()[:, capi.PHASE].clone()

    def after_propagate(self, sim):
        X = sim.prop.last_step(self.W).X
        self.X[self.pos].copy_(X)
        props = sim.wset.properties()
        p1 = props[:, capi.PHASE]
        scale = torch.clamp(torch.cos(props[:, capi.THETA].real), min=0.0)
        ok = (scale > np.finfo(np.float64).tiny) & (self._phase0 != 0)
        ratio = torch.where(ok, p1 / torch.where(ok, self._phase0, torch.ones_like(p1)),
                            torch.zeros_like(p1))
        self.F[self.pos] = torch.where(ok, ratio / torch.where(ok, scale, torch.ones_like(scale)),
                                       torch.zeros_like(p1))
        self.pos = (self.pos + 1) % self.nback

    def after_population_control(self, sim, offspring):
        src = slot_map(offspring)
        moved = np.nonzero(src != np.arange(src.size))[0]
        if moved.size == 0:
            return
        d = torch.as_tensor(moved, device=self.dev)
        s = torch.as_tensor(src[moved], device=self.dev)
        self.X[:, d] = self.X[:, s]
        self.F[:, d] = self.F[:, s]
        for a in self.anchor:
            a[d] = a[s]

    def equilibrated(self, sim, step):
        self._set_anchor(step)

    def measure(self, sim, step):
        bp_step = step - self.bp_pos
        if bp_step < 0:
            raise RuntimeError("back-propagation window starts after the current step")
        if bp_step == self.nback:
            self.samples.append((step, self.estimate(bp_step).cpu().numpy()))
        if bp_step >= self.nback:
            self._set_anchor(step)

    # ---------------------------------------------------------------- the estimate
    def back_propagate(self, nbp):
        """The references propagated backwards through the last nbp stored fields, one copy per
        walker (per spin [nref * W][M][N_s], reference-major, device), and the accumulated log
        det of the re-orthogonalisations [nref * W]."""
        sim = self.sim
        nr, W = self.nref, self.W
        refs = [t.unsqueeze(1).expand(-1, W, -1, -1).reshape(nr * W, self.M, t.shape[2])
                .contiguous() for t in self.trial]
        logdetR = torch.zeros(nr * W, dtype=torch.complex128, device=self.dev)
        slot = self.pos
        for ni in range(nbp - 1, -1, -1):
            slot = (slot - 1) % self.nback
            V = sim.ham.vHS(self.X[slot].contiguous(), sim.dt)
            for s, S in enumerate(refs):
                if S.shape[2] == 0:
                    continue
                Vh = (-V[s % V.shape[0]].conj().transpose(1, 2))
                Vh = (Vh.repeat(nr, 1, 1) if nr > 1 else Vh).contiguous()
                A.det_ops.Propagate(S, self.P1h[s % len(self.P1h)], Vh, self.order)
            if ni == 0 or ni % self.ortho == 0:
                for S in refs:
                    if S.shape[2]:
                        A.det_ops.orthogonalize(S, logdetR)
        return refs, logdetR

    def weights(self, nbp):
        w = self.sim.wset.properties()[:, capi.WEIGHT].clone()
        if self.path_restoration:
            slot = self.pos
            for _ in range(nbp):
                slot = (slot - 1) % self.nback
                w = w * self.F[slot]
        return w

    def estimate(self, nbp):
        """BackPropEstimator.hpp:36-120 and onerdm.hpp: per reference d and walker, the log
        overlap of the back-propagated reference with the anchored walker (both spins; twice the
        one block for CLOSED) plus conj(logdetR_d) after removing its mean over the references
        (doubled for CLOSED), the overlap conj(c_d) e^{that}, each reference's share of the
        walker's total, and sum_w w'_w sum_d share_{w,d} G_{w,d} / sum_w w'_w."""
        refs, logdetR = self.back_propagate(nbp)
        nr, W = self.nref, self.W
        closed = not self.collinear
        L = logdetR.view(nr, W)
        L = L - L.mean(0, keepdim=True)
        if closed:
            L = 2.0 * L
        return reference_onerdm(refs, self.anchor, self.weights(nbp), self.ref_w,
                                torch.conj(L), 2.0 if closed else 1.0)
