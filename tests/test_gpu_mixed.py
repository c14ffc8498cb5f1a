"""Mixed-precision (3xTF32 tcgen05) contractions vs the FP64 oracle.

Tolerances: the 3xTF32 split keeps about 21 significant bits per operand and FP32 accumulation;
the relative (infinity-norm) errors allowed here are 2e-5 for single contractions and 1e-4 for a
full propagation step (several chained products)."""
import numpy as np
import pytest
import torch

from oracle import afqmc as O
from safire_b200.synth import make_workload
from tests.gpu_helpers import make_pair, rand_c, rel_err, to_dev, to_host

pytestmark = pytest.mark.gpu
TOL_ONE = 2e-5
TOL_STEP = 1e-4


@pytest.fixture(scope="module", params=[("cfg1", 128), ("cfg1", 40)])
def case(request, cuda):
    name, W = request.param
    wl = make_workload(name, W=W)
    dham, oham, owfn = make_pair(wl)
    return wl, dham, oham, owfn


def test_vbias_mixed(case):
    from safire_b200 import afqmc as A
    wl, dham, oham, _ = case
    rs = np.random.default_rng(1)
    G = rand_c(rs, wl.W, wl.nup * wl.M, scale=0.3)
    v = torch.zeros((wl.W, wl.Nc), dtype=torch.complex128, device="cuda")
    dham.vbias(to_dev(G), v, wl.dt, precision=A.PREC_MIXED)
    err = rel_err(to_host(v), oham.vbias(G, wl.dt))
    print(f"vbias mixed rel err {err:.2e}")
    assert err < TOL_ONE


def test_vhs_mixed(case):
    from safire_b200 import afqmc as A
    wl, dham, oham, _ = case
    rs = np.random.default_rng(2)
    X = rand_c(rs, wl.W, wl.Nc)
    V = dham.vHS(to_dev(X), wl.dt, precision=A.PREC_MIXED)
    err = rel_err(to_host(V), oham.vHS(X, wl.dt))
    print(f"vHS mixed rel err {err:.2e}")
    assert err < TOL_ONE


def test_energy_mixed(case):
    from safire_b200 import afqmc as A
    wl, dham, oham, _ = case
    rs = np.random.default_rng(3)
    G = rand_c(rs, wl.W, wl.nup * wl.M, scale=0.2)
    E = torch.zeros((wl.W, 3), dtype=torch.complex128, device="cuda")
    dham.energy(E, to_dev(G), precision=A.PREC_MIXED)
    Eo = oham.energy(G)
    Ed = to_host(E)
    errs = [rel_err(Ed[:, q], Eo[:, q]) for q in range(3)]
    print("energy mixed rel errs E1/EXX/EJ", ["%.2e" % e for e in errs])
    assert errs[0] < 1e-12  # E1 stays FP64
    assert max(errs[1:]) < TOL_ONE


def test_step_mixed_vs_fp64(case):
    """One propagation step, same uniforms, FP64 vs mixed: walkers, overlaps, weights."""
    from safire_b200 import afqmc as A
    wl, dham, oham, owfn = case
    W = wl.W
    res = {}
    for prec in (A.PREC_FP64, A.PREC_MIXED):
        ws = A.WalkerSet(wl.walker_type, wl.M, wl.nup, wl.ndn, W)
        ws.init_from_trial(dham)
        wfn = A.NOMSD(dham)
        wfn.Energy(ws, set_properties=True)
        torch.cuda.synchronize()
        e = sum(ws.getProperty(p) for p in (A.capi.E1, A.capi.EXX, A.capi.EJ))
        ws.setProperty(A.capi.PSEUDO_ELOC, e)
        prop = A.Propagator(dham, A.default_params(dt=wl.dt, precision=prec), W)
        u = O.HostRandomGenerator(O.split_seed(0, 0, 1)).sample_uniform(W * wl.Nc)
        ud = to_dev(u.reshape(W, wl.Nc), torch.float64)
        for _ in range(3):
            prop.Propagate(ws, -30.0, ud)
        torch.cuda.synchronize()
        res[prec] = (to_host(ws.SlaterMatrices(0)), to_host(ws.properties()))
    S64, p64 = res[A.PREC_FP64]
    Smx, pmx = res[A.PREC_MIXED]
    eS = rel_err(Smx, S64)
    eO = rel_err(pmx[:, O.OVLP], p64[:, O.OVLP])
    eW = rel_err(pmx[:, O.WEIGHT], p64[:, O.WEIGHT])
    print(f"3 steps mixed vs fp64: S {eS:.2e} ovlp {eO:.2e} weight {eW:.2e}")
    assert eS < TOL_STEP and eO < TOL_STEP and eW < TOL_STEP


def test_mixed_no_device_timeout(case):
    """The tensor-core kernels' bounded waits never ran out in the calls above."""
    from safire_b200 import afqmc as A
    wl, dham, _, _ = case
    G = torch.zeros((wl.W, wl.nup * wl.M), dtype=torch.complex128, device="cuda")
    v = torch.zeros((wl.W, wl.Nc), dtype=torch.complex128, device="cuda")
    dham.vbias(G, v, wl.dt, precision=A.PREC_MIXED)
    assert dham.device_error_flag() == 0


def test_energy_mixed_large_block(cuda):
    """The fused exchange kernel at N = 50 electrons (the benchmark's block size), M = 200."""
    from safire_b200 import afqmc as A
    wl = make_workload("cfg2", W=5, Nc=48)
    dham, oham, _ = make_pair(wl)
    rs = np.random.default_rng(4)
    G = rand_c(rs, 5, wl.nup * wl.M, scale=0.1)
    E = torch.zeros((5, 3), dtype=torch.complex128, device="cuda")
    dham.energy(E, to_dev(G), precision=A.PREC_MIXED)
    Eo = oham.energy(G)
    Ed = to_host(E)
    errs = [rel_err(Ed[:, q], Eo[:, q]) for q in range(3)]
    print("energy mixed N=50 rel errs", ["%.2e" % e for e in errs])
    assert max(errs[1:]) < TOL_ONE
    assert dham.device_error_flag() == 0


def test_exchange_single_tf32_error(cuda):
    """Plain-TF32 exchange (one product per real product): error reported against FP64."""
    from safire_b200 import afqmc as A
    wl = make_workload("cfg2", W=6, Nc=64)
    dham, oham, _ = make_pair(wl)
    dham.set_exchange_split(1)
    rs = np.random.default_rng(5)
    G = rand_c(rs, 6, wl.nup * wl.M, scale=0.1)
    E = torch.zeros((6, 3), dtype=torch.complex128, device="cuda")
    dham.energy(E, to_dev(G), precision=A.PREC_MIXED)
    Eo = oham.energy(G)
    Ed = to_host(E)
    errs = [rel_err(Ed[:, q], Eo[:, q]) for q in range(1, 3)]
    print("energy 1xTF32 exchange rel errs EXX/EJ", ["%.2e" % e for e in errs])
    assert max(errs) < 2e-3
    dham.set_exchange_split(3)


def _mixed_steps(wl, dham, fused, nsteps=2, order=None, split_format=1):
    from safire_b200 import afqmc as A
    W = wl.W
    dham.set_split_format(split_format)
    dham.set_taylor_fused(fused)
    ws = A.WalkerSet(wl.walker_type, wl.M, wl.nup, wl.ndn, W)
    ws.init_from_trial(dham)
    kw = {} if order is None else {"taylor_n": order}
    prop = A.Propagator(dham, A.default_params(dt=wl.dt, precision=A.PREC_MIXED, **kw), W)
    u = O.HostRandomGenerator(O.split_seed(0, 0, 7)).sample_uniform(W * wl.Nc)
    ud = to_dev(u.reshape(W, wl.Nc), torch.float64)
    for _ in range(nsteps):
        prop.Propagate(ws, -30.0, ud)
    torch.cuda.synchronize()
    dham.set_taylor_fused(1)
    dham.set_split_format(0)
    return to_host(ws.SlaterMatrices(0)), to_host(ws.properties())


@pytest.mark.parametrize("mode", [3, 6])
@pytest.mark.parametrize("name,W,Nc,order", [("cfg1", 300, None, None), ("cfg1", 20, None, 0),
                                             ("cfg2", 6, 40, None), ("cfg1", 301, None, 3)])
def test_taylor_fused_vs_per_term(cuda, name, W, Nc, order, mode):
    """The persistent Taylor kernel (all products of a walker in one CTA; mode 2 / 3: one / two
    walkers in flight per CTA; 6: one in flight with the running sum in tensor memory) against
    one GEMM launch per product: the same split arithmetic (the TF32 split, one accumulator),
    different kernels; W = 300, 301 run several walkers per CTA (301: one slot ends early).  The
    modes with a second accumulator for the small products (2, 4) sum differently, more
    accurately, and are checked against complex128 below.  The FP16 split of the fused kernel is checked against complex128
    in test_gpu_mixed_full.py and below."""
    kw = {"W": W} if Nc is None else {"W": W, "Nc": Nc}
    wl = make_workload(name, **kw)
    dham, _, _ = make_pair(wl)
    Sf, pf = _mixed_steps(wl, dham, mode, order=order)
    Su, pu = _mixed_steps(wl, dham, 0, order=order)
    eS = rel_err(Sf, Su)
    eO = rel_err(pf[:, O.OVLP], pu[:, O.OVLP])
    print(f"fused ({mode}) vs per-term Taylor ({name}, W={W}, order={order}): S {eS:.2e} "
          f"ovlp {eO:.2e}")
    assert eS < 1e-5 and eO < 1e-5
    assert dham.device_error_flag() == 0


def test_autotune_leaves_the_run_unchanged(cuda):
    """The autotuner times every Taylor variant on the live walkers and restores them: a run that
    autotunes and one that is set to the chosen variant by hand take bit-identical next steps."""
    import torch
    from safire_b200 import afqmc as A
    from safire_b200.driver import RunParams, Simulation
    from safire_b200.synth import make_workload
    wl = make_workload("cfg2", W=64)
    runs = []
    for tune in (True, False):
        sim = Simulation.from_workload(wl, W=64, precision=A.PREC_MIXED,
                                       rp=RunParams(equilibration_steps=0, seed=3))
        sim.step()
        sim.step()
        before = sim.wset.buffer.clone()
        if tune:
            best, ms = sim.autotune()
            assert best in (2, 4) and all(t > 0 for t in ms.values()), (best, ms)
            assert set(ms) == {0, 2, 3, 4, 5, 6, 7}  # FP16 variants are tried on these shapes
            assert torch.equal(sim.wset.buffer, before)
            chosen = best
        else:
            sim.ham.set_taylor_fused(chosen)
        sim._g_ready = False
        sim.step()
        runs.append(sim.wset.buffer.clone())
    assert torch.equal(runs[0], runs[1])


def test_tile_candidates_are_bit_identical(cuda):
    """Every tile choice the tile autotuner picks among gives the same results bit for bit:
    vbias with 128- and 64-wide tiles, the exchange energy with every L2 block size; and the
    autotuner leaves the walkers as they were."""
    import torch
    from safire_b200 import afqmc as A
    from safire_b200.driver import RunParams, Simulation
    from safire_b200.synth import make_workload
    wl = make_workload("cfg2", W=160, Nc=400)
    sim = Simulation.from_workload(wl, W=160, precision=A.PREC_MIXED,
                                   rp=RunParams(equilibration_steps=0, seed=5))
    sim.step()
    G, _ = sim.wfn.MixedDensityMatrix(sim.wset)
    outs_v, outs_e = [], []
    for bn, blk in [(128, 64), (64, 16), (128, 32), (64, 128)]:
        sim.ham.set_tiles(bn, blk)
        v = torch.zeros((160, wl.Nc), dtype=torch.complex128, device="cuda")
        sim.ham.vbias(G, v, wl.dt, precision=A.PREC_MIXED)
        E = torch.zeros((160, 3), dtype=torch.complex128, device="cuda")
        sim.ham.energy(E, G, precision=A.PREC_MIXED)
        outs_v.append(v)
        outs_e.append(E)
    for v, E in zip(outs_v[1:], outs_e[1:]):
        assert torch.equal(v, outs_v[0])
        assert torch.equal(E, outs_e[0])
    before = sim.wset.buffer.clone()
    tiles, ms = sim.autotune_tiles()
    print("tile autotuner:", tiles, {k: round(t, 3) for k, t in ms.items()})
    assert tiles["vbias_bn"] in (64, 128) and tiles["exchange_block"] in (16, 32, 64, 128)
    assert tiles["vhs_symmetric"] in (0, 1)
    assert torch.equal(sim.wset.buffer, before)
    assert sim.ham.get_tiles() == (tiles["vbias_bn"], tiles["exchange_block"])


@pytest.mark.parametrize("mode", [2, 4, 5, 7])
@pytest.mark.parametrize("name,W,Nc,order", [("cfg1", 300, None, None), ("cfg1", 20, None, 0),
                                             ("cfg1", 301, None, 3)])
def test_taylor_fused_fp16_vs_fp64(cuda, name, W, Nc, order, mode):
    """The persistent Taylor kernel with a second accumulator for the small split products (2:
    TF32 split, 4: FP16 split) and in the FP16 split (4, 5, 7; operands and every term scaled by
    powers of two) against complex128 propagation on the same walkers and fields: walkers within
    the one-step bound of the mixed path (1e-4), log-overlaps within 1e-3 (the log-det sums the
    walkers' error over the electrons)."""
    from safire_b200 import afqmc as A
    kw = {"W": W} if Nc is None else {"W": W, "Nc": Nc}
    wl = make_workload(name, **kw)
    dham, _, _ = make_pair(wl)
    Sf, pf = _mixed_steps(wl, dham, mode, order=order, split_format=1 if mode == 2 else 2)
    ws = A.WalkerSet(wl.walker_type, wl.M, wl.nup, wl.ndn, W)
    ws.init_from_trial(dham)
    kwp = {} if order is None else {"taylor_n": order}
    prop = A.Propagator(dham, A.default_params(dt=wl.dt, **kwp), W)
    u = O.HostRandomGenerator(O.split_seed(0, 0, 7)).sample_uniform(W * wl.Nc)
    ud = to_dev(u.reshape(W, wl.Nc), torch.float64)
    for _ in range(2):
        prop.Propagate(ws, -30.0, ud)
    S64, p64 = to_host(ws.SlaterMatrices(0)), to_host(ws.properties())
    eS = rel_err(Sf, S64)
    eO = float(np.max(np.abs(pf[:, O.OVLP] - p64[:, O.OVLP])))
    print(f"fused ({mode}) vs complex128 ({name}, W={W}, order={order}): S {eS:.2e} "
          f"log-ovlp {eO:.2e}")
    assert eS < TOL_STEP and eO < 1e-3
    assert dham.device_error_flag() == 0
