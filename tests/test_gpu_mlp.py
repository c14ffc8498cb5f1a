"""The control-variate network's BF16 tensor-core kernels through the C ABI: predictions and
gradients against the oracle's statement with the same rounding points, training on a smooth
target, the feature kernel, and the multi-fidelity exchange estimate on a running simulation."""
import numpy as np
import pytest
import torch

from oracle import mlp as O
from tests.gpu_helpers import rel_err

pytestmark = pytest.mark.gpu


def _case(seed, D, H, B):
    rs = np.random.default_rng(seed)
    n = H * D + H + H * H + H + H + 1
    p = (rs.standard_normal(n) * 0.3).astype(np.float32)
    X = (rs.standard_normal((B, D)) * 2 + 0.5).astype(np.float32)
    t = rs.standard_normal(B).astype(np.float32) * 3 - 1
    mean = (rs.standard_normal(D) * 0.3).astype(np.float32)
    istd = (0.5 + rs.random(D)).astype(np.float32)
    return p, X, t, mean, istd


@pytest.mark.parametrize("D,H,B", [(10, 8, 7), (96, 64, 130), (3300, 512, 256)])
def test_predict_and_gradients_vs_oracle(cuda, D, H, B):
    from safire_b200.mlp import ExchangeMLP
    p, X, t, mean, istd = _case(D, D, H, B)
    net = ExchangeMLP(D, H, seed=1)
    net.set_params(p)
    net.set_normalization(mean, istd, 0.7, 2.5)
    Xd, td = torch.as_tensor(X, device=cuda), torch.as_tensor(t, device=cuda)
    y = net.predict(Xd).cpu().numpy()
    yo, loss_o, g_o = O.loss_and_grad_bf16(p, X, t, D, H, mean, istd, 0.7, 2.5)
    assert rel_err(y, yo * 2.5 + 0.7) < 2e-3
    loss = float(net.gradients(Xd, td).item())
    assert abs(loss - loss_o) < 2e-3 * abs(loss_o)
    g = net.params(1)
    assert rel_err(g, g_o) < 2e-3
    # each parameter block on its own (a wrong transpose would hide in the norm of W1)
    o = 0
    for size in (H * D, H, H * H, H, H, 1):
        assert rel_err(g[o:o + size], g_o[o:o + size]) < 5e-3, (o, size)
        o += size


def test_training_reduces_loss(cuda):
    """A smooth function of the features is learned: the loss falls by an order of magnitude."""
    from safire_b200.mlp import ExchangeMLP
    rs = np.random.default_rng(0)
    D, n = 64, 8192
    X = rs.standard_normal((n, D)).astype(np.float32)
    y = (np.sin(X[:, 0]) + 0.5 * X[:, 1] * X[:, 2] + 0.2 * X[:, 3:10].sum(1)).astype(np.float32)
    Xd, yd = torch.as_tensor(X, device=cuda), torch.as_tensor(y, device=cuda)
    net = ExchangeMLP(D, 128, seed=2)
    net.fit_normalization(Xd, yd)
    hist = net.fit(Xd, yd, epochs=40, batch=512, lr=2e-3)
    assert hist[-1] < 0.1 * hist[0], hist[::8]
    pred = net.predict(Xd).cpu().numpy()
    assert np.sqrt(np.mean((pred - y) ** 2)) < 0.3 * np.std(y)


def test_exchange_features(cuda):
    from safire_b200.mlp import exchange_features
    rs = np.random.default_rng(1)
    W, Nc, N, M = 5, 17, 4, 9
    v = torch.as_tensor(rs.standard_normal((W, Nc)) + 1j * rs.standard_normal((W, Nc)),
                        device=cuda)
    G = torch.as_tensor(rs.standard_normal((W, N * M + 3)) + 1j * rs.standard_normal((W, N * M + 3)),
                        device=cuda)
    X = exchange_features(v, G, N, M).cpu().numpy()
    vh, Gh = v.cpu().numpy(), G.cpu().numpy()
    d = np.stack([Gh[:, a * M + a] for a in range(N)], 1)
    ref = np.concatenate([vh.real, vh.imag, d.real, d.imag], 1).astype(np.float32)
    assert np.array_equal(X, ref)
    E = torch.as_tensor(rs.standard_normal((W, 3)) + 1j * rs.standard_normal((W, 3)), device=cuda)
    XE = exchange_features(v, G, N, M, E).cpu().numpy()
    Eh = E.cpu().numpy()
    extra = np.stack([Eh[:, 0].real, Eh[:, 0].imag, Eh[:, 2].real, Eh[:, 2].imag], 1)
    assert np.array_equal(XE, np.concatenate([ref, extra.astype(np.float32)], 1))


def test_control_variate_on_a_run(cuda):
    """Pairs from the exact kernel during equilibration train the network; afterwards the
    multi-fidelity exchange (exact on 1/8 of the walkers) stays unbiased (checked over many
    random subsets of the same walkers) and has a much smaller spread than subsampling alone."""
    from safire_b200.driver import RunParams, Simulation
    from safire_b200.mlp import ExchangeControlVariate
    from safire_b200.synth import make_workload
    wl = make_workload("cfg1", W=256)
    sim = Simulation.from_workload(wl, W=256, rp=RunParams(equilibration_steps=1000, seed=0))
    cv = ExchangeControlVariate(sim, hidden=256, fraction=1 / 8, seed=0)
    for step in range(60):
        sim.step(measure=False)
        if step % 2 == 0:
            cv.collect()
    hist = cv.fit(epochs=60, batch=512, lr=1e-3)
    assert hist[-1] < 0.3 * hist[0], hist[::10]
    for _ in range(5):
        sim.step(measure=False)
    ests, exact = [], None
    for _ in range(64):
        _, o = cv.measure(exact=exact is None)
        if exact is None:
            exact = o["exx_exact"]
            # the Coulomb term from the force bias equals the energy kernel's
            assert abs(o["ej_from_vbias"] - o["ej_exact"]) < 1e-10 * abs(o["ej_exact"])
        ests.append(o["exx_mf"].real)
    ests = np.array(ests)
    # unbiased: the mean over subsets agrees with the exact value within its standard error
    se = ests.std(ddof=1) / np.sqrt(ests.size)
    assert abs(ests.mean() - exact.real) < 4 * se + 1e-9 * abs(exact.real)
    # variance reduction against plain subsampling (network output zero)
    from safire_b200 import capi
    w = sim.wset.properties()[:, capi.WEIGHT].real.cpu().numpy()
    G, _ = sim.wfn.MixedDensityMatrix(sim.wset)
    E = torch.empty((sim.wset.W, 3), dtype=torch.complex128, device=G.device)
    sim.ham.energy(E, G, addH1=False, addEJ=False, addEXX=True)
    e = E[:, 1].real.cpu().numpy()
    rs = np.random.default_rng(5)
    plain = [O.multifidelity_sum(w, np.zeros_like(e), e[S], S) / w.sum()
             for S in (np.sort(rs.choice(e.size, 32, replace=False)) for _ in range(64))]
    assert ests.std() < 0.5 * np.std(plain), (ests.std(), np.std(plain))


def test_control_variate_leading_cholesky(cuda):
    """The low-fidelity base EXX_k over the leading Cholesky vectors: with all Nc vectors it is the
    exact exchange, and the estimate equals the exact one for any subset; with Nc / 8 vectors the
    estimate stays unbiased over random subsets and beats subsampling on the remainder alone."""
    from safire_b200 import capi
    from safire_b200.driver import RunParams, Simulation
    from safire_b200.mlp import ExchangeControlVariate, lowrank_hamiltonian
    from safire_b200.synth import make_workload
    wl = make_workload("cfg1", W=128)
    args = (wl.walker_type, wl.M, wl.nup, wl.ndn, wl.Likn, wl.hij, wl.E0, wl.PsiT)
    sim = Simulation.from_workload(wl, W=128, rp=RunParams(equilibration_steps=1000, seed=3))
    for _ in range(20):
        sim.step(measure=False)
    for k, tol in ((wl.Nc, 1e-9), (wl.Nc // 8, None)):
        cv = ExchangeControlVariate(sim, hidden=128, fraction=1 / 8, seed=0,
                                    lowrank=lowrank_hamiltonian(args, k))
        assert cv.mlp.D == 2 * wl.Nc + 2 * wl.nup + 2
        for _ in range(6):
            sim.step(measure=False)
            cv.collect()
        cv.fit(epochs=20, batch=256, lr=1e-3)
        ests, exact = [], None
        for _ in range(48):
            _, o = cv.measure(exact=exact is None)
            exact = o["exx_exact"] if exact is None else exact
            ests.append(o["exx_mf"].real)
        ests = np.array(ests)
        if tol is not None:
            assert np.all(np.abs(ests - exact.real) < tol * abs(exact.real)), (ests[:4], exact)
            continue
        se = ests.std(ddof=1) / np.sqrt(ests.size)
        assert abs(ests.mean() - exact.real) < 4 * se + 1e-9 * abs(exact.real)
        w = sim.wset.properties()[:, capi.WEIGHT].real.cpu().numpy()
        G, _ = sim.wfn.MixedDensityMatrix(sim.wset)
        E = torch.empty((sim.wset.W, 3), dtype=torch.complex128, device=G.device)
        sim.ham.energy(E, G, addH1=False, addEJ=False, addEXX=True)
        e = E[:, 1].real.cpu().numpy()
        rs = np.random.default_rng(5)
        plain = [O.multifidelity_sum(w, np.zeros_like(e), e[S], S) / w.sum()
                 for S in (np.sort(rs.choice(e.size, 16, replace=False)) for _ in range(48))]
        assert ests.std() < 0.5 * np.std(plain), (ests.std(), np.std(plain))
