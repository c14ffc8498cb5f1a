"""run_afqmc-style step loop over the C ABI (src/AFQMC/execute.cpp:106-209,
src/AFQMC/Drivers/run_afqmc.cpp:69-113).

The per-step work (G, vbias, fields, vHS, propagation, overlaps, phaseless update) is one C-ABI
call, afqmc_prop_step; this module only sequences steps, orthogonalisation, comb population
control and energy measurements at the reference's cadence, and keeps Eshift.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import torch

from . import afqmc as A
from .capi import E1, EJ, EXX, OVLP, PSEUDO_ELOC


@dataclass
class RunParams:
    walker_ortho_interval: int = 5
    population_control_interval: int = 10
    measure_interval: int = 10
    equilibration_steps: int = 100
    seed: int = 0


@dataclass
class Simulation:
    ham: A.HamiltonianOperations
    wfn: A.NOMSD
    wset: A.WalkerSet
    prop: A.Propagator
    walker_rng: A.HostRandomGenerator
    rp: RunParams
    dt: float
    Eshift: float
    relax: float
    precision: int = A.PREC_FP64
    step_index: int = 0
    energies: list = field(default_factory=list)

    @staticmethod
    def from_workload(wl, W=None, precision=A.PREC_FP64, rp=None, **prop_kw):
        rp = rp or RunParams()
        W = W or wl.W
        ham = A.HamiltonianOperations(wl.walker_type, wl.M, wl.nup, wl.ndn, wl.Likn, wl.hij,
                                      wl.E0, wl.PsiT)
        wfn = A.NOMSD(ham)
        wset = A.WalkerSet(wl.walker_type, wl.M, wl.nup, wl.ndn, W)
        wset.init_from_trial(ham)
        walker_rng = A.HostRandomGenerator(A.split_seed(rp.seed, 0, 0))
        # initial energy, seeded pseudo energy and Eshift (execute.cpp:171-184)
        wfn.Energy(wset, set_properties=True, precision=precision)
        torch.cuda.synchronize()
        e1, exx, ej = (wset.getProperty(p) for p in (E1, EXX, EJ))
        wset.setProperty(PSEUDO_ELOC, e1 + exx + ej)
        w = wset.getProperty(0)
        Eshift = float((np.sum(w * (e1 + exx + ej)) / np.sum(w)).real)
        params = A.default_params(dt=wl.dt, precision=precision, **prop_kw)
        prop = A.Propagator(ham, params, W)
        prop.set_field_seed(A.split_seed(rp.seed, 0, 1))
        n = rp.equilibration_steps
        relax = 1 - math.exp(-10.0 / n) if n > 1 else 1.0
        return Simulation(ham, wfn, wset, prop, walker_rng, rp, wl.dt, Eshift, relax, precision)

    def average_pseudo_energy(self):
        s = A.pseudo_energy_sums(self.wset, self.dt)
        s = s.cpu().numpy()
        return math.log((s[0] / s[1]).real) / self.dt

    def measure(self):
        E, _ = self.wfn.Energy(self.wset, set_properties=False, precision=self.precision)
        sums = A.energy_sums(self.wset, E).cpu().numpy()
        energy = float((np.sum(sums[:3]) / sums[3]).real)
        return energy, sums, E

    def step(self, uniforms=None, measure=True):
        """One iteration of the run_afqmc loop.  Returns the measured energy or None."""
        step = self.step_index
        self.prop.Propagate(self.wset, self.Eshift, uniforms)
        if step % self.rp.walker_ortho_interval == 0:
            self.prop.Orthogonalize(self.wset)
        if step % self.rp.population_control_interval == 0:
            A.population_control(self.wset, self.walker_rng)
        out = None
        if step >= self.rp.equilibration_steps:
            if measure and step % self.rp.measure_interval == 0:
                out, _, _ = self.measure()
                self.energies.append((step, out))
        else:
            self.Eshift += self.relax * (self.average_pseudo_energy() - self.Eshift)
        self.step_index += 1
        return out
