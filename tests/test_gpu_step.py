"""Per-step parity of the full walker step (FP64) against the oracle, fed the same field uniforms
(the reference's DEVICE_RNG_FROM_HOST mode) and the same walker RNG."""
import math

import numpy as np
import pytest
import torch

from oracle import afqmc as O
from safire_b200.synth import make_workload
from tests.gpu_helpers import rel_err, to_dev, to_host

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _wrap_diff(a, b, period):
    d = np.asarray(a) - np.asarray(b)
    return d - period * np.round(d / period)


def _cmp_complex_mod(a, b, period):
    """relative error with the imaginary parts compared modulo `period` (branch of a log)."""
    a = np.asarray(a)
    b = np.asarray(b)
    re = rel_err(a.real, b.real)
    im = np.max(np.abs(_wrap_diff(a.imag, b.imag, period))) / max(1.0, np.max(np.abs(b)))
    return max(re, im)


@pytest.mark.parametrize("W,steps", [(16, 12)])
def test_step_parity_fp64(cuda, W, steps):
    from safire_b200 import afqmc as A
    from safire_b200.driver import RunParams, Simulation

    wl = make_workload("cfg1", W=W)
    rp = RunParams(equilibration_steps=5, seed=0)
    sim = Simulation.from_workload(wl, W=W, rp=rp)

    # oracle set-up in the same order as execute.cpp
    oham = O.Real3IndexFactorization(wl.walker_type, wl.M, wl.nup, wl.ndn, wl.Likn, wl.hij, wl.E0,
                                     wl.PsiT)
    owfn = O.NOMSD(oham, wl.PsiT)
    ows = O.WalkerSet.from_trial(owfn, W)
    E, ov = owfn.Energy(ows.SA, ows.SB)
    ows.props[:, O.OVLP] = ov
    ows.props[:, O.E1], ows.props[:, O.EXX], ows.props[:, O.EJ] = E[:, 0], E[:, 1], E[:, 2]
    ows.props[:, O.PSEUDO_ELOC] = E.sum(axis=1)
    Eshift_o = O.average_energy(ows)
    oprop = O.Propagator(owfn, O.PropagatorParams(dt=wl.dt))
    walker_rng = O.HostRandomGenerator(O.split_seed(0, 0, 0))
    field_rng = O.HostRandomGenerator(O.split_seed(0, 0, 1))
    relax = 1 - math.exp(-10.0 / rp.equilibration_steps)

    assert abs(sim.Eshift - Eshift_o) < 1e-10 * abs(Eshift_o)
    props0 = to_host(sim.wset.properties())
    assert _cmp_complex_mod(props0[:, O.PSEUDO_ELOC], ows.props[:, O.PSEUDO_ELOC], 1e300) < TOL

    for step in range(steps):
        u = field_rng.sample_uniform(W * wl.Nc).reshape(W, wl.Nc)
        # device step
        sim.prop.Propagate(sim.wset, sim.Eshift, to_dev(u, torch.float64))
        last = sim.prop.last_step(W)
        # oracle step
        oprop.propagate(ows, Eshift_o, u)
        lo = oprop.last
        assert rel_err(to_host(last.vbias), lo["vbias"]) < TOL, step
        assert rel_err(to_host(last.X), lo["X"]) < TOL, step
        assert rel_err(to_host(last.HW), lo["HW"]) < TOL, step
        assert rel_err(to_host(last.mf), lo["mf"]) < TOL, step
        assert _cmp_complex_mod(to_host(last.new_ovlp), lo["new_ov"], 2 * np.pi) < TOL, step
        SA = to_host(sim.wset.SlaterMatrices(0))
        assert rel_err(SA, ows.SA) < TOL, step
        props = to_host(sim.wset.properties())
        assert rel_err(props[:, O.WEIGHT], ows.props[:, O.WEIGHT]) < TOL, step
        assert rel_err(props[:, O.PHASE], ows.props[:, O.PHASE]) < TOL, step
        assert _cmp_complex_mod(props[:, O.PSEUDO_ELOC], ows.props[:, O.PSEUDO_ELOC],
                                2 * np.pi / wl.dt) < TOL, step

        if step % rp.walker_ortho_interval == 0:
            sim.prop.Orthogonalize(sim.wset)
            oprop.orthogonalize(ows)
            assert rel_err(to_host(sim.wset.SlaterMatrices(0)), ows.SA) < TOL, step
        if step % rp.population_control_interval == 0:
            off_d = A.population_control(sim.wset, sim.walker_rng)
            off_o = O.population_control_single_rank(walker_rng, ows)
            assert np.array_equal(off_d, off_o), step  # comb branching bit-exact
            props = to_host(sim.wset.properties())
            assert rel_err(props[:, O.WEIGHT], ows.props[:, O.WEIGHT]) < TOL, step
            assert rel_err(to_host(sim.wset.SlaterMatrices(0)), ows.SA) < TOL, step
        if step >= rp.equilibration_steps:
            if step % rp.measure_interval == 0:
                e_d, sums, Ed = sim.measure()
                m = O.energy_measure(owfn, ows)
                assert rel_err(to_host(Ed), m["E"]) < TOL, step
                assert abs(e_d - m["energy"]) < TOL * abs(m["energy"]), step
        else:
            sim.Eshift += sim.relax * (sim.average_pseudo_energy() - sim.Eshift)
            Eshift_o += relax * (O.average_pseudo_energy(ows, wl.dt) - Eshift_o)
            assert abs(sim.Eshift - Eshift_o) < TOL * abs(Eshift_o), step
        sim.step_index += 1

    stats = sim.prop.bound_stats()
    assert stats[0] == oprop.eloc_stats.total
    assert stats[1] == oprop.eloc_stats.upper and stats[2] == oprop.eloc_stats.lower


def test_step_parity_fp64_full_size(cuda):
    """The benchmark system itself (M=200, N=50+50, Nc=1600): 40 FP64 steps with
    orthogonalisation, comb and Eshift relaxation track the oracle walker for walker."""
    from safire_b200 import afqmc as A
    from safire_b200.driver import RunParams, Simulation

    W, steps = 4, 40
    wl = make_workload("cfg2", W=W)
    rp = RunParams(equilibration_steps=100, seed=0)
    sim = Simulation.from_workload(wl, W=W, rp=rp)
    oham = O.Real3IndexFactorization(wl.walker_type, wl.M, wl.nup, wl.ndn, wl.Likn, wl.hij, wl.E0,
                                     wl.PsiT)
    owfn = O.NOMSD(oham, wl.PsiT)
    ows = O.WalkerSet.from_trial(owfn, W)
    E, ov = owfn.Energy(ows.SA, ows.SB)
    ows.props[:, O.OVLP] = ov
    ows.props[:, O.E1], ows.props[:, O.EXX], ows.props[:, O.EJ] = E[:, 0], E[:, 1], E[:, 2]
    ows.props[:, O.PSEUDO_ELOC] = E.sum(axis=1)
    Eshift_o = O.average_energy(ows)
    oprop = O.Propagator(owfn, O.PropagatorParams(dt=wl.dt))
    walker_rng = O.HostRandomGenerator(O.split_seed(0, 0, 0))
    field_rng = O.HostRandomGenerator(O.split_seed(0, 0, 1))
    relax = 1 - math.exp(-10.0 / rp.equilibration_steps)
    for step in range(steps):
        u = field_rng.sample_uniform(W * wl.Nc).reshape(W, wl.Nc)
        sim.prop.Propagate(sim.wset, sim.Eshift, to_dev(u, torch.float64))
        oprop.propagate(ows, Eshift_o, u)
        if step % rp.walker_ortho_interval == 0:
            sim.prop.Orthogonalize(sim.wset)
            oprop.orthogonalize(ows)
        if step % rp.population_control_interval == 0:
            off_d = A.population_control(sim.wset, sim.walker_rng)
            off_o = O.population_control_single_rank(walker_rng, ows)
            assert np.array_equal(off_d, off_o), step
        sim.Eshift += sim.relax * (sim.average_pseudo_energy() - sim.Eshift)
        Eshift_o += relax * (O.average_pseudo_energy(ows, wl.dt) - Eshift_o)
        sim.step_index += 1
        props = to_host(sim.wset.properties())
        assert rel_err(to_host(sim.wset.SlaterMatrices(0)), ows.SA) < TOL, step
        assert rel_err(props[:, O.WEIGHT], ows.props[:, O.WEIGHT]) < TOL, step
        assert _cmp_complex_mod(props[:, O.PSEUDO_ELOC], ows.props[:, O.PSEUDO_ELOC],
                                2 * np.pi / wl.dt) < TOL, step
        assert abs(sim.Eshift - Eshift_o) < TOL * abs(Eshift_o), step


def test_device_rng_step_runs(cuda):
    """The production path: fields from the device Philox generator, full loop with measurement."""
    from safire_b200.driver import RunParams, Simulation
    wl = make_workload("cfg1", W=32)
    sim = Simulation.from_workload(wl, W=32, rp=RunParams(equilibration_steps=3))
    for _ in range(14):
        sim.step()
    torch.cuda.synchronize()
    props = to_host(sim.wset.properties())
    assert np.all(np.isfinite(props))
    assert len(sim.energies) == 1
    e = sim.energies[0][1]
    assert np.isfinite(e) and -40 < e < -20


def test_nonfinite_walker_is_dropped(cuda):
    """A walker whose local energy is not finite gets weight 0 and keeps its old eloc
    (WalkerSetUpdate.hpp:127-133).  The fault is injected on the host into the walker data."""
    from safire_b200.driver import RunParams, Simulation
    wl = make_workload("cfg1", W=8)
    sim = Simulation.from_workload(wl, W=8, rp=RunParams(equilibration_steps=100))
    old = sim.wset.getProperty(O.PSEUDO_ELOC)
    ov = sim.wset.getProperty(O.OVLP)
    ov[3] = complex(np.inf, 0)  # old overlap infinite -> eloc = -inf
    sim.wset.setProperty(O.OVLP, ov)
    sim.prop.Propagate(sim.wset, sim.Eshift)
    torch.cuda.synchronize()
    w = sim.wset.getProperty(O.WEIGHT)
    el = sim.wset.getProperty(O.PSEUDO_ELOC)
    assert w[3] == 0 and el[3] == old[3]
    assert np.all(w[[0, 1, 2, 4, 5, 6, 7]] != 0)


@pytest.mark.parametrize("precision", [0, 1])
def test_graph_step_matches_eager(cuda, precision):
    """The CUDA-graph replay of a step (device fields, Eshift from device memory) gives the same
    walkers, weights and energies as launching the step eagerly, bit for bit."""
    from safire_b200.driver import RunParams, Simulation
    wl = make_workload("cfg1", W=24)
    sims = []
    for g in (False, True):
        sim = Simulation.from_workload(wl, W=24, precision=precision,
                                       rp=RunParams(equilibration_steps=6))
        sim.use_graph = g
        sims.append(sim)
    for _ in range(14):
        for sim in sims:
            sim.step()
    torch.cuda.synchronize()
    # steps 1..13 replay graphs: one per flag set (after orthogonalisation / comb the density
    # matrix is recomputed, otherwise reused)
    assert sims[1].graph is not None and len(sims[1].graph.graphs) == 2
    assert sims[1].graph.kernels_replayed() > 0
    a, b = (to_host(s.wset.buffer) for s in sims)
    assert np.array_equal(a, b)
    assert sims[0].energies == sims[1].energies
    assert sims[0].Eshift == sims[1].Eshift


@pytest.mark.parametrize("precision", [0, 1])
def test_graph_step_with_given_fields_matches_eager(cuda, precision):
    """Fields given on the device: the replayed step (its field buffer refilled before each
    replay) equals the eager step, bit for bit."""
    from safire_b200.driver import RunParams, Simulation
    wl = make_workload("cfg1", W=24)
    rs = np.random.default_rng(4)
    U = torch.as_tensor(rs.random((14, 24, wl.Nc)), device="cuda")
    sims = []
    for g in (False, True):
        sim = Simulation.from_workload(wl, W=24, precision=precision,
                                       rp=RunParams(equilibration_steps=6))
        sim.use_graph = g
        sims.append(sim)
    for k in range(14):
        for sim in sims:
            sim.step(U[k])
    torch.cuda.synchronize()
    assert sims[1].graph_u is not None and sims[1].graph_u.kernels_replayed() > 0
    a, b = (to_host(s.wset.buffer) for s in sims)
    assert np.array_equal(a, b)
    assert sims[0].energies == sims[1].energies


@pytest.mark.parametrize("precision", [0, 1])
def test_density_reuse_matches_recompute(cuda, precision):
    """Steps that keep the propagated walkers' density matrix for the next step (skipped
    recomputation between orthogonalisations / combs) give the same run as recomputing it at
    every step."""
    from safire_b200.driver import RunParams, Simulation
    wl = make_workload("cfg1", W=24)
    sims = []
    for reuse in (False, True):
        sim = Simulation.from_workload(wl, W=24, precision=precision,
                                       rp=RunParams(equilibration_steps=6))
        sim.reuse_density = reuse
        sims.append(sim)
    for _ in range(23):
        for sim in sims:
            sim.step()
    torch.cuda.synchronize()
    a, b = (to_host(s.wset.buffer) for s in sims)
    assert rel_err(a, b) < 1e-13
    assert np.allclose([e for _, e in sims[0].energies], [e for _, e in sims[1].energies],
                       rtol=1e-13, atol=0)
