"""Learned exchange-energy control variate (no reference counterpart).

An MLP maps each walker's features (its force bias vbias and the diagonal of its compact mixed
density matrix) to its exchange energy.  It is trained by the library's own BF16 tensor-core
kernels (safire_b200/csrc/mlp.cu) on (features, exact exchange) pairs that the exact kernel
produces during equilibration.  A measurement then evaluates the network on every walker and the
exact exchange (Real3IndexFactorization energy_impl, Real3IndexFactorization.hpp:476-590) on a
uniform random subset, combined as

    sum_w omega_w EX_w  ~  sum_w omega_w f_w + (W / k) sum_{s in S} omega_s (EX_s - f_s),

which is unbiased over the subset whatever the network predicts: the exact kernel stays the reference
value and the network only reduces the variance of the subsampled estimate.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import afqmc as A
from . import capi
from .capi import call, vp


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _s(stream):
    return A._stream(stream)


class ExchangeMLP:
    """features (D) -> H -> H -> 1, GELU; parameters FP32 on the device."""

    def __init__(self, D, H=512, seed=0):
        h = vp()
        call("afqmc_mlp_create", int(D), int(H), int(seed), C.byref(h))
        self.handle, self.D, self.H = h, int(D), int(H)
        self.n_params = int(capi.lib().afqmc_mlp_num_params(h))
        self._loss = torch.zeros(1, dtype=torch.float32, device="cuda")

    def __del__(self):
        h = getattr(self, "handle", None)
        try:
            if h and capi._lib is not None:
                capi._lib.afqmc_mlp_destroy(h)
        except (AttributeError, TypeError):  # interpreter shutdown: the library is gone
            pass
        self.handle = None

    def set_normalization(self, mean, istd, y_mean, y_std):
        m = np.ascontiguousarray(mean, dtype=np.float32)
        s = np.ascontiguousarray(istd, dtype=np.float32)
        call("afqmc_mlp_set_normalization", self.handle, A._host_ptr(m), A._host_ptr(s),
             float(y_mean), float(y_std))
        self.norm = (m, s, float(y_mean), float(y_std))

    def fit_normalization(self, X, y):
        """Standardise with the statistics of training features X [n][D] and targets y [n]."""
        Xh = X.double()
        mean = Xh.mean(0)
        std = Xh.std(0)
        istd = torch.where(std > 1e-12, 1.0 / std, torch.ones_like(std))
        yh = y.double()
        self.set_normalization(mean.cpu().numpy(), istd.cpu().numpy(), float(yh.mean()),
                               float(max(yh.std(), 1e-12)))

    def params(self, which=0):
        out = np.zeros(self.n_params, dtype=np.float32)
        call("afqmc_mlp_params", self.handle, int(which), A._host_ptr(out), 0)
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        call("afqmc_mlp_params", self.handle, 0, A._host_ptr(p), 1)

    def predict(self, X, out=None, stream=None):
        X = X.contiguous()
        out = out if out is not None else torch.empty(X.shape[0], dtype=torch.float32,
                                                      device=X.device)
        call("afqmc_mlp_predict", self.handle, _p(X), int(X.shape[0]), _p(out), _s(stream))
        return out

    def gradients(self, X, t, stream=None):
        X, t = X.contiguous(), t.contiguous()
        call("afqmc_mlp_gradients", self.handle, _p(X), _p(t), int(X.shape[0]), _p(self._loss),
             _s(stream))
        return self._loss

    def train_step(self, X, t, lr, stream=None):
        X, t = X.contiguous(), t.contiguous()
        call("afqmc_mlp_train_step", self.handle, _p(X), _p(t), int(X.shape[0]), float(lr),
             _p(self._loss), _s(stream))
        return self._loss

    def fit(self, X, y, epochs=20, batch=1024, lr=1e-3, seed=0):
        """Adam over shuffled mini-batches; returns the mean loss of every epoch (host)."""
        g = torch.Generator(device="cpu").manual_seed(seed)
        n = X.shape[0]
        hist = []
        for _ in range(epochs):
            perm = torch.randperm(n, generator=g).to(X.device)
            tot, nb = 0.0, 0
            for i in range(0, n - batch + 1 if n >= batch else 1, batch):
                idx = perm[i:i + batch]
                tot += float(self.train_step(X[idx], y[idx], lr).item())
                nb += 1
            hist.append(tot / max(nb, 1))
        return hist


def exchange_features(vbias, G, N, M, E=None, stream=None):
    """X [W][2 Nc + 2 N (+ 4 with E)] (FP32) from vbias [W][Nc], the compact density matrix
    G [W][..] and optionally the walkers' E1 and EJ (E [W][3])."""
    W, Nc = vbias.shape
    D = 2 * Nc + 2 * N + (4 if E is not None else 0)
    X = torch.empty((W, D), dtype=torch.float32, device=vbias.device)
    call("afqmc_exchange_features", _p(vbias), int(vbias.stride(0)), _p(G), int(G.stride(0)),
         int(N), int(M), int(Nc), int(W), _p(E), _p(X), _s(stream))
    return X


def lowrank_hamiltonian(ham_args, k):
    """A HamiltonianOperations over the first k Cholesky vectors: ham_args = (walker_type, M, nup,
    ndn, Likn [nspin_H2][M][M][Nc], hij, E0, PsiT) as HamiltonianOperations takes them."""
    walker_type, M, nup, ndn, Likn, hij, E0, PsiT = ham_args
    return A.HamiltonianOperations(walker_type, M, nup, ndn,
                                   np.ascontiguousarray(np.asarray(Likn)[..., :k]), hij, E0, PsiT)


class ExchangeControlVariate:
    """Multi-fidelity exchange energy for a Simulation (safire_b200.driver): collect pairs during
    equilibration, fit, then measure with the exact exchange on a random fraction of walkers."""

    def __init__(self, sim, hidden=512, fraction=1.0 / 8, seed=0, scalars=False,
                 sampling="uniform", lowrank=None):
        """scalars: also feed each walker's E1 and EJ to the network.  sampling: "uniform" (k
        distinct walkers) or "weight" (k draws with probability |w| / sum |w|, with replacement:
        the correction is then a Horvitz-Thompson sum, still unbiased, and concentrates the exact
        evaluations on the walkers that carry the estimate).  lowrank: an optional
        HamiltonianOperations over the leading Cholesky vectors (lowrank_hamiltonian); its
        exchange energy EXX_k of every walker (real and imaginary parts) is a further feature and
        the network learns the remainder EXX - EXX_k, so the prediction is EXX_k + network."""
        self.sampling = sampling
        self.sim = sim
        ham = sim.ham
        self.N, self.M, self.Nc = ham.nup, ham.M, ham.Nc
        self.nel = ham.nel
        self.scalars = scalars
        self.lowrank = lowrank
        D = 2 * self.Nc + 2 * self.N + (4 if scalars else 0) + (2 if lowrank else 0)
        self.mlp = ExchangeMLP(D, hidden, seed)
        self.fraction = fraction
        self._seed = seed
        self._gen = None  # device generator of the exact-evaluation draws
        self.X, self.y = [], []
        dev = sim.wset.buffer.device
        self._v = torch.empty((sim.wset.W, self.Nc), dtype=torch.complex128, device=dev)

    def _features(self):
        """G of the walkers, their vbias, E1 and EJ (E [W][3], EXX left zero) and the features.
        EJ comes from the Coulomb vector the force bias already holds (Kl = vbias / (sqrt(dt) a)
        with a = 2 for CLOSED walkers and EJ = sclj / 2 sum_n Kl^2 with sclj = a^2): EJ =
        sum_n vbias_n^2 / (2 dt) for either walker type."""
        sim = self.sim
        G, _ = sim.wfn.MixedDensityMatrix(sim.wset)
        sim.ham.vbias(G, self._v, sim.dt, precision=sim.precision)
        E = torch.empty((sim.wset.W, 3), dtype=torch.complex128, device=G.device)
        sim.ham.energy(E, G, addH1=True, addEJ=False, addEXX=False, precision=sim.precision)
        E[:, 2] = (self._v * self._v).sum(1) / (2.0 * sim.dt)
        X = exchange_features(self._v, G, self.N, self.M, E if self.scalars else None)
        base = None
        if self.lowrank is not None:
            Ek = torch.empty_like(E)
            self.lowrank.energy(Ek, G, addH1=False, addEJ=False, addEXX=True,
                                precision=sim.precision)
            base = Ek[:, 1]
            X = torch.cat([X, torch.view_as_real(base).float()], 1)
        return G, E, X, base

    def collect(self):
        """One training sample per walker: features and the exact exchange energy (less the
        leading-vector exchange with lowrank)."""
        G, _, X, base = self._features()
        E = torch.empty((self.sim.wset.W, 3), dtype=torch.complex128, device=G.device)
        self.sim.ham.energy(E, G, addH1=False, addEJ=False, addEXX=True,
                            precision=self.sim.precision)
        self.X.append(X)
        y = E[:, 1] if base is None else E[:, 1] - base
        self.y.append(y.real.float())

    def fit(self, epochs=30, batch=1024, lr=1e-3):
        X = torch.cat(self.X)
        y = torch.cat(self.y)
        self.mlp.fit_normalization(X, y)
        return self.mlp.fit(X, y, epochs=epochs, batch=min(batch, X.shape[0]), lr=lr)

    def measure(self, exact=False):
        """Mixed-estimator energy with the multi-fidelity exchange (exact=True: every walker's
        exact exchange).  Returns (energy, {'exx_mf', 'exx_exact' (when computed)})."""
        sim = self.sim
        W = sim.wset.W
        # E1 and EJ exactly for every walker
        G, E, X, base = self._features()
        dev = G.device
        w = sim.wset.properties()[:, capi.WEIGHT]
        f = self.mlp.predict(X).double()
        if base is not None:
            f = base + f
        k = max(1, int(round(self.fraction * W)))
        # the draws stay on the device (no host round trip between the launches)
        if self._gen is None or self._gen.device != dev:
            self._gen = torch.Generator(device=dev)
            self._gen.manual_seed(self._seed)
        if self.sampling == "weight":
            aw = w.abs()
            prob = aw / aw.sum()
            S = torch.multinomial(prob, k, replacement=True, generator=self._gen)
            # sum over the draws of w_s (e_s - f_s) / (k p_s); a walker drawn twice is evaluated
            # twice
            scale = 1.0 / (k * prob[S])
        else:
            S = torch.randperm(W, device=dev, generator=self._gen)[:k]
            scale = torch.full((k,), W / k, dtype=torch.float64, device=dev)
        Es = torch.empty((S.numel(), 3), dtype=torch.complex128, device=dev)
        sim.ham.energy(Es, G[S].contiguous(), addH1=False, addEJ=False, addEXX=True,
                       precision=sim.precision)
        ex_mf = (w * f).sum() + (scale * w[S] * (Es[:, 1] - f[S])).sum()
        wsum = w.sum()
        e_other = (w * (E[:, 0] + E[:, 2])).sum()
        energy = ((e_other + ex_mf) / wsum).real
        out = {"exx_mf": complex((ex_mf / wsum).item())}  # the first host read: all is enqueued
        if exact:
            Ea = torch.empty((W, 3), dtype=torch.complex128, device=dev)
            sim.ham.energy(Ea, G, addH1=True, addEJ=True, addEXX=True, precision=sim.precision)
            out["exx_exact"] = complex(((w * Ea[:, 1]).sum() / wsum).item())
            out["ej_exact"] = complex(((w * Ea[:, 2]).sum() / wsum).item())
            out["ej_from_vbias"] = complex(((w * E[:, 2]).sum() / wsum).item())
        return float(energy.item()), out
