"""run_afqmc-style step loop over the C ABI (src/AFQMC/execute.cpp:106-209,
src/AFQMC/Drivers/run_afqmc.cpp:69-113).  Under an initialised torch.distributed process group
each rank holds its own walkers: the energy and pseudo-energy sums are summed over the ranks and
population control is the distributed comb (safire_b200.population).

The per-step work (G, vbias, fields, vHS, propagation, overlaps, phaseless update) is one C-ABI
call, afqmc_prop_step; this module only sequences steps, orthogonalisation, comb population
control and energy measurements at the reference's cadence, and keeps Eshift.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import torch
import torch.distributed as dist

from . import afqmc as A
from .capi import E1, EJ, EXX, OVLP, PSEUDO_ELOC


def _world():
    return dist.get_world_size() if dist.is_available() and dist.is_initialized() else 1


def _rank():
    return dist.get_rank() if _world() > 1 else 0


def _sum_over_ranks(t):
    """In-place sum over the ranks of a device (NCCL) or host (gloo) tensor."""
    if _world() > 1:
        if dist.get_backend() == "nccl":
            dist.all_reduce(t)
        else:
            h = t.cpu()
            dist.all_reduce(h)
            t.copy_(h)
    return t


@dataclass
class RunParams:
    walker_ortho_interval: int = 5
    population_control_interval: int = 10  # 0: none inside step()
    measure_interval: int = 10
    equilibration_steps: int = 100
    seed: int = 0


class StepGraph:
    """The propagation step (afqmc_prop_step_flags) captured in CUDA graphs, one per flag set.

    Eshift is read from a one-element device buffer (`eshift`, refreshed before each replay), so
    equilibration can keep moving it; the fields come from the device Philox generator (its
    counter lives on the device and advances inside the graph), or from a fixed device buffer
    `uniforms` [W, Nc] that the caller refills before each replay.  Capture records without
    executing, so it is done after the first eager step (every buffer allocated) and does not
    advance the run."""

    def __init__(self, prop, wset, eshift, uniforms=None):
        self.prop, self.wset, self.eshift, self.uniforms = prop, wset, eshift, uniforms
        self.graphs, self.kernels = {}, {}
        self.replayed = 0

    def _capture(self, flags):
        stream = torch.cuda.Stream()
        stream.wait_stream(torch.cuda.current_stream())
        g = torch.cuda.CUDAGraph()
        n0 = A.lib().afqmc_kernel_launches()
        with torch.cuda.graph(g, stream=stream):
            self.prop.Propagate_flags(self.wset, self.eshift, self.uniforms, flags)
        # kernels recorded in the graph (the library counts launches as it records them)
        self.kernels[flags] = A.lib().afqmc_kernel_launches() - n0
        torch.cuda.current_stream().wait_stream(stream)
        self.graphs[flags] = g

    def replay(self, flags):
        if flags not in self.graphs:
            self._capture(flags)
        self.graphs[flags].replay()
        self.replayed += self.kernels[flags]

    def kernels_replayed(self):
        return self.replayed


def _initial_state(wfn, wset, precision):
    """Initial energies, overlaps and seeded pseudo energies of the walkers, and Eshift
    (execute.cpp:171-184)."""
    wfn.Energy(wset, set_properties=True, precision=precision)
    torch.cuda.synchronize()
    e1, exx, ej = (wset.getProperty(p) for p in (E1, EXX, EJ))
    wset.setProperty(PSEUDO_ELOC, e1 + exx + ej)
    w = wset.getProperty(0)
    sums = torch.tensor([np.sum(w * (e1 + exx + ej)), np.sum(w)], dtype=torch.complex128,
                        device=wset.buffer.device)
    sums = _sum_over_ranks(sums).cpu().numpy()
    return float((sums[0] / sums[1]).real)


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
    use_graph: bool = False
    graph: StepGraph = None
    graph_u: StepGraph = None  # the captured step for fields given on the device
    _u_buf: torch.Tensor = None
    # the step leaves the density matrix of the propagated walkers for the next step, which
    # skips recomputing it unless orthogonalisation or population control changed the walkers
    reuse_density: bool = True
    # estimators that follow the walkers between measurements (safire_b200.backprop): each has
    # before_step, after_propagate, after_population_control(sim, offspring), equilibrated(sim,
    # step) and measure(sim, step), called at the points of the run_afqmc loop they name
    observers: list = field(default_factory=list)
    # host field stream (use_host_fields); None: the device generator
    field_rng: A.HostRandomGenerator = None
    _g_ready: bool = False
    _eshift_dev: torch.Tensor = None

    @staticmethod
    def from_workload(wl, W=None, precision=A.PREC_FP64, rp=None, trial=None, vMF=None,
                      multidet=None, ham=None, **prop_kw):
        """wl: a safire_b200.synth.Workload.  trial: an optional PHMSD trial
        (safire_b200.synth.PHMSDTrial, COLLINEAR workload whose PsiT is its reference
        determinant); multidet: an optional several-determinant NOMSD trial (PsiTs, ci) with
        PsiTs[d] the per-spin PsiT of determinant d (wl.PsiT is determinant 0's); vMF: the mean
        field [Nc] (host) of either, default determinant 0's.  ham: the Hamiltonian operations
        to use instead of the workload's Cholesky ones (a THC HamiltonianOperations.thc over
        the same system; one determinant)."""
        rp = rp or RunParams()
        W = W or wl.W
        if ham is not None and (trial is not None or multidet is not None):
            raise ValueError("a given Hamiltonian takes a single-determinant trial")
        if ham is None:
            ham = A.HamiltonianOperations(wl.walker_type, wl.M, wl.nup, wl.ndn, wl.Likn, wl.hij,
                                          wl.E0, wl.PsiT)
        ph = None
        if trial is not None and multidet is not None:
            raise ValueError("a PHMSD trial and a several-determinant NOMSD trial exclude each other")
        if trial is not None:
            ph = A.PHMSD(trial)
            ph.set_hamiltonian(wl.Likn, wl.hij, wl.E0)
            wfn = A.PHMSDWavefunction(ph)
        elif multidet is not None:
            PsiTs, ci = multidet
            hams = [ham] + [A.HamiltonianOperations(wl.walker_type, wl.M, wl.nup, wl.ndn, wl.Likn,
                                                    wl.hij, wl.E0, P) for P in PsiTs[1:]]
            ph = wfn = A.NOMSDMulti(hams, ci)
        else:
            wfn = A.NOMSD(ham)
        wset = A.WalkerSet(wl.walker_type, wl.M, wl.nup, wl.ndn, W)
        wset.init_from_trial(ham)
        # the comb's generator is the same on every rank (the reference's root draws it); the
        # auxiliary fields of each rank's walkers come from that rank's own stream
        walker_rng = A.HostRandomGenerator(A.split_seed(rp.seed, 0, 0))
        Eshift = _initial_state(wfn, wset, precision)
        params = A.default_params(dt=wl.dt, precision=precision, **prop_kw)
        prop = A.Propagator(ham, params, W)
        prop.set_field_seed(A.split_seed(rp.seed, _rank(), 1))
        if ph is not None:
            prop.set_trial(ph, vMF)
        n = rp.equilibration_steps
        relax = 1 - math.exp(-10.0 / n) if n > 1 else 1.0
        sim = Simulation(ham, wfn, wset, prop, walker_rng, rp, wl.dt, Eshift, relax, precision)
        if ph is not None:
            sim.reuse_density = False  # the multi-determinant step recomputes its density matrix
        return sim

    def restart(self):
        """Walkers back at the trial with unit weights, their energies and overlaps, a re-seeded
        Eshift and step counter; the field and walker generators continue their streams."""
        self.wset.init_from_trial(self.ham)
        self.Eshift = _initial_state(self.wfn, self.wset, self.precision)
        self.step_index = 0
        self._g_ready = False

    def use_host_fields(self):
        """Draw every step's field uniforms on the host from std::mt19937 seeded with
        split_seed(seed, rank, 1) and uniform_real_distribution<double>, W x Nc per step in
        walker-major order: the field stream of the reference's host build (execute.cpp:124-125,
        Random.hpp:37-51, AFQMCBasePropagator.cpp:706-716), so a seeded run reproduces the
        reference's own.  Steps with host fields are launched eagerly, not from a graph."""
        self.field_rng = A.HostRandomGenerator(A.split_seed(self.rp.seed, _rank(), 1))

    def autotune(self):
        """Let the library pick the fastest step variant for these walkers (mixed precision);
        the walkers are left as they were.  Returns (mode, {mode: step ms})."""
        best, ms = self.prop.autotune(self.wset)
        self._g_ready = False
        self.graph = self.graph_u = None  # a captured step holds the previous variant's kernels
        return best, ms

    def autotune_tiles(self):
        """Let the library pick the tile shapes / orders with bit-identical results (vbias tile
        width, vHS form, exchange L2 block) for these walkers; the walkers are left as they
        were.  Returns ({choice: value}, {candidate: ms})."""
        out = self.prop.autotune_tiles(self.wset)
        self._g_ready = False
        self.graph = self.graph_u = None  # a captured step holds the previous tiles' kernels
        return out

    def average_pseudo_energy(self):
        s = _sum_over_ranks(A.pseudo_energy_sums(self.wset, self.dt))
        s = s.cpu().numpy()
        return math.log((s[0] / s[1]).real) / self.dt

    def measure(self):
        E, _ = self.wfn.Energy(self.wset, set_properties=False, precision=self.precision)
        sums = _sum_over_ranks(A.energy_sums(self.wset, E)).cpu().numpy()
        energy = float((np.sum(sums[:3]) / sums[3]).real)
        return energy, sums, E

    def step(self, uniforms=None, measure=True):
        """One iteration of the run_afqmc loop.  Returns the measured energy or None."""
        step = self.step_index
        if self._eshift_dev is None:
            self._eshift_dev = torch.zeros(1, dtype=torch.float64, device=self.wset.buffer.device)
        self._eshift_dev.fill_(float(self.Eshift))
        for o in self.observers:
            o.before_step(self)
        if uniforms is None and self.field_rng is not None:
            W, Nc = self.wset.W, self.ham.Nc
            u = self.field_rng.sample_uniform(W * Nc).reshape(W, Nc)
            uniforms = torch.as_tensor(u, device=self.wset.buffer.device)
        flags = 0
        if self.reuse_density:
            flags = A.capi.STEP_KEEP_G | (A.capi.STEP_G_READY if self._g_ready else 0)
        if self.use_graph and uniforms is None and (step > 0 or self.graph is not None):
            # device fields: replay the captured step (captured on first use, after the first
            # eager step has allocated every buffer; a restart keeps the captured graphs)
            if self.graph is None:
                self.graph = StepGraph(self.prop, self.wset, self._eshift_dev)
            self.graph.replay(flags)
        elif (self.use_graph and uniforms is not None and uniforms.is_cuda
              and (step > 0 or self.graph_u is not None)):
            # fields given on the device: a second captured step reads them from a fixed buffer,
            # refilled here (a device copy on the step's stream)
            if self.graph_u is None:
                self._u_buf = torch.empty_like(uniforms)
                self.graph_u = StepGraph(self.prop, self.wset, self._eshift_dev, self._u_buf)
            self._u_buf.copy_(uniforms)
            self.graph_u.replay(flags)
        else:
            self.prop.Propagate_flags(self.wset, self._eshift_dev, uniforms, flags)
        self._g_ready = self.reuse_density
        for o in self.observers:
            o.after_propagate(self)
        if step % self.rp.walker_ortho_interval == 0:
            self.prop.Orthogonalize(self.wset)
            self._g_ready = False
        pci = self.rp.population_control_interval
        if pci > 0 and step % pci == 0:  # 0: the caller controls the population itself
            self._g_ready = False
            if _world() > 1:
                if self.observers:
                    raise NotImplementedError("walker-following estimators run on one rank")
                from .population import population_control_distributed
                population_control_distributed(self.wset, self.walker_rng)
            else:
                off = A.population_control(self.wset, self.walker_rng)
                for o in self.observers:
                    o.after_population_control(self, off)
        out = None
        if step >= self.rp.equilibration_steps:
            if measure and step % self.rp.measure_interval == 0:
                out, _, _ = self.measure()
                self.energies.append((step, out))
            for o in self.observers:
                o.measure(self, step)
        else:
            self.Eshift += self.relax * (self.average_pseudo_energy() - self.Eshift)
            if step == self.rp.equilibration_steps - 1:
                for o in self.observers:
                    o.equilibrated(self, step)
        self.step_index += 1
        return out
