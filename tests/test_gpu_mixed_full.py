"""Mixed precision against complex128 at the benchmark's own shapes: M=200, N=50+50 (CLOSED),
N_chol=1600, 256 walkers, fixed auxiliary fields.

256 walkers exceed the 148 SMs, so the persistent tensor-core kernels (exchange, Taylor) hold
several walkers per CTA, and the Taylor kernel's two-walkers-in-flight mode runs with its second
slot busy.  Each quantity is compared three ways: mixed vs the library's complex128 path on all
256 walkers, and both against the oracle (a CPU restatement of Real3IndexFactorization and the
propagator, Real3IndexFactorization.hpp:282-428, 476-590; AFQMCBasePropagator.cpp:289-392) on
the first four walkers.

Every mixed-precision check runs with both operand formats of the split: TF32 terms and FP16
terms of operands scaled by powers of two (afqmc_ham_set_split_format); both keep 22 significant
bits per operand.

Bounds (relative, infinity norm over the compared array):
  - complex128 vs oracle: 1e-10, the parity bar of the FP64 path;
  - single mixed contraction (vbias, vHS, EXX, EJ): 2e-5.  The 3xTF32 split keeps ~21 bits of
    each operand (the dropped lo x lo product is 2^-22 relative); FP32 accumulation over K =
    1600 (vHS) or 1000-element K slices (vbias, whose slices are summed in FP64) adds ~sqrt(K)
    2^-24;
  - one mixed propagation step (vbias -> fields -> vHS -> six Taylor terms -> overlap ->
    weight): 1e-4 on the walkers and on the phaseless angles; 1e-3 absolute on the real part of
    the new log-overlaps and relative on the weights.  The log-overlap log det(PsiT S) of a
    50-electron walker sums the walker's relative error (~4e-6) over its 50 columns, amplified
    by the conditioning of PsiT S (measured: 2.6e-4), and the phaseless weight moves by exactly
    that log-overlap difference (exp(-dt (eloc - Eshift)), eloc holding -log(ov ratio) / dt).
"""
import numpy as np
import pytest
import torch

from oracle import afqmc as O
from safire_b200.synth import make_workload
from tests.gpu_helpers import make_pair, rel_err, to_dev, to_host

pytestmark = pytest.mark.gpu
W = 256
NO = 4  # walkers checked against the oracle
TOL_FP64 = 1e-10
TOL_ONE = 2e-5
TOL_STEP = 1e-4
TOL_LOGOV = 1e-3


@pytest.fixture(scope="module")
def full(cuda):
    """The benchmark system with 256 walkers taken two complex128 steps away from the trial
    (so every walker differs), as a walker buffer to start each test from."""
    from safire_b200 import afqmc as A
    wl = make_workload("cfg2", W=W)
    dham, oham, owfn = make_pair(wl)
    ws = A.WalkerSet(wl.walker_type, wl.M, wl.nup, wl.ndn, W)
    ws.init_from_trial(dham)
    A.NOMSD(dham).Energy(ws, set_properties=True)
    torch.cuda.synchronize()
    e = sum(ws.getProperty(p) for p in (A.capi.E1, A.capi.EXX, A.capi.EJ))
    ws.setProperty(A.capi.PSEUDO_ELOC, e)
    eshift = float(np.mean(e).real)
    prop = A.Propagator(dham, A.default_params(dt=wl.dt), W)
    rng = O.HostRandomGenerator(O.split_seed(11, 0, 1))
    for _ in range(2):
        u = rng.sample_uniform(W * wl.Nc).reshape(W, wl.Nc)
        prop.Propagate(ws, eshift, to_dev(u, torch.float64))
    torch.cuda.synchronize()
    del prop
    u = rng.sample_uniform(W * wl.Nc).reshape(W, wl.Nc)  # the fields of the compared step
    return dict(wl=wl, dham=dham, oham=oham, owfn=owfn, buf=ws.buffer.clone(), eshift=eshift,
                u=u)


def _scale_bias(mx, ref):
    """Systematic part of a mixed result: s - 1 for the least-squares scale s with mx ~ s ref.
    A rounding that is unbiased gives |s - 1| far below the elementwise error; an accumulation
    that truncates toward zero gives s < 1."""
    mx, ref = np.asarray(mx).ravel(), np.asarray(ref).ravel()
    return float(np.real(np.vdot(ref, mx)) / np.real(np.vdot(ref, ref)) - 1.0)


def _walkers(f):
    from safire_b200 import afqmc as A
    wl = f["wl"]
    ws = A.WalkerSet(wl.walker_type, wl.M, wl.nup, wl.ndn, W)
    ws.buffer.copy_(f["buf"])
    torch.cuda.synchronize()
    return ws


def _G(f):
    from safire_b200 import afqmc as A
    G, _ = A.NOMSD(f["dham"]).MixedDensityMatrix(_walkers(f))
    torch.cuda.synchronize()
    return G


FORMATS = pytest.mark.parametrize("fmt", [1, 2], ids=["tf32", "fp16"])


@pytest.fixture
def fmt_set(full, fmt):
    """Select the split format for one test and restore the automatic choice afterwards."""
    assert full["dham"].set_split_format(fmt) == (fmt == 2)
    yield fmt
    full["dham"].set_split_format(0)


@FORMATS
def test_full_vbias(full, fmt_set):
    from safire_b200 import afqmc as A
    wl, dham, oham = full["wl"], full["dham"], full["oham"]
    G = _G(full)
    out = {}
    for prec in (A.PREC_FP64, A.PREC_MIXED):
        v = torch.zeros((W, wl.Nc), dtype=torch.complex128, device="cuda")
        dham.vbias(G, v, wl.dt, precision=prec)
        out[prec] = to_host(v)
    vo = oham.vbias(to_host(G)[:NO], wl.dt)
    e64 = rel_err(out[A.PREC_FP64][:NO], vo)
    emx = rel_err(out[A.PREC_MIXED], out[A.PREC_FP64])
    emo = rel_err(out[A.PREC_MIXED][:NO], vo)
    print(f"vbias W={W} fmt {fmt_set}: fp64 vs oracle {e64:.2e}, mixed vs fp64 {emx:.2e}, "
          f"mixed vs oracle {emo:.2e}, scale bias "
          f"{_scale_bias(out[A.PREC_MIXED], out[A.PREC_FP64]):.2e}")
    assert e64 < TOL_FP64
    assert emx < TOL_ONE and emo < TOL_ONE
    assert dham.device_error_flag() == 0


@FORMATS
def test_full_vhs(full, fmt_set):
    from safire_b200 import afqmc as A
    wl, dham, oham = full["wl"], full["dham"], full["oham"]
    # fixed fields shaped like the step's: N(0,1) real parts, small force-bias imaginary parts
    rs = np.random.default_rng(21)
    X = rs.standard_normal((W, wl.Nc)) + 0.05j * rs.standard_normal((W, wl.Nc))
    Xd = to_dev(X)
    V64 = to_host(dham.vHS(Xd, wl.dt, precision=A.PREC_FP64))
    Vmx = to_host(dham.vHS(Xd, wl.dt, precision=A.PREC_MIXED))
    Vo = oham.vHS(X[:NO], wl.dt)
    e64 = rel_err(V64[0, :NO], Vo.reshape(V64[0, :NO].shape))
    emx = rel_err(Vmx, V64)
    emo = rel_err(Vmx[0, :NO], Vo.reshape(V64[0, :NO].shape))
    print(f"vHS W={W} fmt {fmt_set}: fp64 vs oracle {e64:.2e}, mixed vs fp64 {emx:.2e}, "
          f"mixed vs oracle {emo:.2e}, scale bias {_scale_bias(Vmx, V64):.2e}")
    assert e64 < TOL_FP64
    assert emx < TOL_ONE and emo < TOL_ONE
    assert dham.device_error_flag() == 0


@FORMATS
def test_full_vhs_symmetric_form(full, fmt_set):
    """The symmetric tensor-core vHS (the i <= k pairs only, mirrored in the epilogue; the
    benchmark's Cholesky vectors are symmetric) against the contraction over all M^2 pairs:
    the same products, summed in the same order, so they agree to the last bit of the split
    planes' rounding."""
    from safire_b200 import afqmc as A
    wl, dham = full["wl"], full["dham"]
    rs = np.random.default_rng(22)
    X = to_dev(rs.standard_normal((W, wl.Nc)) + 0.05j * rs.standard_normal((W, wl.Nc)))
    assert dham.set_vhs_symmetry(True)
    Vs = to_host(dham.vHS(X, wl.dt, precision=A.PREC_MIXED))
    assert not dham.set_vhs_symmetry(False)
    Vf = to_host(dham.vHS(X, wl.dt, precision=A.PREC_MIXED))
    dham.set_vhs_symmetry(True)
    e = rel_err(Vs, Vf)
    asym = rel_err(Vs, np.swapaxes(Vs, -1, -2))
    print(f"vHS symmetric vs all pairs: {e:.2e}; V - V^T {asym:.2e}")
    assert e < 1e-6 and asym == 0.0
    assert dham.device_error_flag() == 0


@FORMATS
def test_full_energy(full, fmt_set):
    from safire_b200 import afqmc as A
    wl, dham, oham = full["wl"], full["dham"], full["oham"]
    G = _G(full)
    out = {}
    for prec in (A.PREC_FP64, A.PREC_MIXED):
        E = torch.zeros((W, 3), dtype=torch.complex128, device="cuda")
        dham.energy(E, G, precision=prec)
        out[prec] = to_host(E)
    Eo = oham.energy(to_host(G)[:NO])
    for q, name in ((1, "EXX"), (2, "EJ")):
        e64 = rel_err(out[A.PREC_FP64][:NO, q], Eo[:, q])
        emx = rel_err(out[A.PREC_MIXED][:, q], out[A.PREC_FP64][:, q])
        emo = rel_err(out[A.PREC_MIXED][:NO, q], Eo[:, q])
        print(f"{name} W={W} fmt {fmt_set}: fp64 vs oracle {e64:.2e}, mixed vs fp64 {emx:.2e}, "
              f"mixed vs oracle {emo:.2e}, scale bias "
              f"{_scale_bias(out[A.PREC_MIXED][:, q], out[A.PREC_FP64][:, q]):.2e}")
        assert e64 < TOL_FP64
        assert emx < TOL_ONE and emo < TOL_ONE
    # E1 stays complex128 in both
    assert rel_err(out[A.PREC_MIXED][:, 0], out[A.PREC_FP64][:, 0]) < 1e-12
    assert dham.device_error_flag() == 0


def _angle_err(a, b):
    d = np.angle(np.exp(1j * (np.asarray(a) - np.asarray(b))))
    return float(np.max(np.abs(d)))


@FORMATS
@pytest.mark.parametrize("mode", [0, 2, 3, 4, 5, 6, 7])
def test_full_step(full, mode, fmt_set):
    """One propagation step from the same walkers with the same field uniforms: complex128 vs
    mixed with the Taylor series as per-term GEMMs (0) or the persistent kernel with one (2, 4,
    6, 7) or two (3, 5) walkers in flight per CTA, in the TF32 split (2, 3, 6) or the FP16 split
    (4, 5, 7, which fall back to TF32 under the TF32 split format)."""
    from safire_b200 import afqmc as A
    wl, dham, owfn = full["wl"], full["dham"], full["owfn"]
    u = full["u"]
    res = {}
    for prec in (A.PREC_FP64, A.PREC_MIXED):
        ws = _walkers(full)
        if prec == A.PREC_MIXED:
            dham.set_taylor_fused(mode)
        prop = A.Propagator(dham, A.default_params(dt=wl.dt, precision=prec), W)
        prop.Propagate(ws, full["eshift"], to_dev(u, torch.float64))
        last = prop.last_step(W)
        res[prec] = dict(S=to_host(ws.SlaterMatrices(0)), props=to_host(ws.properties()),
                         vbias=to_host(last.vbias), X=to_host(last.X),
                         ov=to_host(last.new_ovlp))
        del prop
    dham.set_taylor_fused(1)
    r64, rmx = res[A.PREC_FP64], res[A.PREC_MIXED]

    # oracle step on the first walkers, same buffer and uniforms
    buf = to_host(full["buf"])
    MN = wl.M * wl.nup
    ows = O.WalkerSet(buf[:NO, :MN].reshape(NO, wl.M, wl.nup).copy(), None,
                      buf[:NO, MN:MN + O.NPROP].copy(), NO, wl.walker_type)
    oprop = O.Propagator(owfn, O.PropagatorParams(dt=wl.dt))
    oprop.propagate(ows, full["eshift"], u[:NO])
    lo = oprop.last

    assert rel_err(r64["S"][:NO], ows.SA) < TOL_FP64
    assert rel_err(r64["vbias"][:NO], lo["vbias"]) < TOL_FP64
    assert rel_err(r64["props"][:NO, O.WEIGHT], ows.props[:, O.WEIGHT]) < TOL_FP64

    e = {
        "S_scale_bias": _scale_bias(rmx["S"], r64["S"]),
        "vbias": rel_err(rmx["vbias"], r64["vbias"]),
        "X": rel_err(rmx["X"], r64["X"]),
        "S": rel_err(rmx["S"], r64["S"]),
        "S_oracle": rel_err(rmx["S"][:NO], ows.SA),
        "weight": rel_err(rmx["props"][:, O.WEIGHT], r64["props"][:, O.WEIGHT]),
        "log_ovlp_re": float(np.max(np.abs(rmx["ov"].real - r64["ov"].real))),
        "log_ovlp_im": _angle_err(rmx["ov"].imag, r64["ov"].imag),
        "phase": _angle_err(np.angle(rmx["props"][:, O.PHASE]),
                            np.angle(r64["props"][:, O.PHASE])),
    }
    print(f"step W={W} taylor mode {mode} fmt {fmt_set}: " +
          ", ".join(f"{k} {v:.2e}" for k, v in e.items()))
    assert e["vbias"] < TOL_ONE and e["X"] < TOL_ONE
    assert e["S"] < TOL_STEP and e["S_oracle"] < TOL_STEP and e["weight"] < TOL_LOGOV
    assert e["log_ovlp_re"] < TOL_LOGOV and e["log_ovlp_im"] < TOL_STEP
    assert e["phase"] < TOL_STEP
    assert dham.device_error_flag() == 0


def test_full_fp16_vs_tf32(full):
    """The two split formats against each other on the same inputs: vbias, vHS and the exchange
    agree to the split precision (both within 2e-5 of complex128)."""
    from safire_b200 import afqmc as A
    wl, dham = full["wl"], full["dham"]
    G = _G(full)
    rs = np.random.default_rng(23)
    X = to_dev(rs.standard_normal((W, wl.Nc)) + 0.05j * rs.standard_normal((W, wl.Nc)))
    out = {}
    for fmt in (1, 2):
        dham.set_split_format(fmt)
        v = torch.zeros((W, wl.Nc), dtype=torch.complex128, device="cuda")
        dham.vbias(G, v, wl.dt, precision=A.PREC_MIXED)
        V = dham.vHS(X, wl.dt, precision=A.PREC_MIXED)
        E = torch.zeros((W, 3), dtype=torch.complex128, device="cuda")
        dham.energy(E, G, precision=A.PREC_MIXED)
        out[fmt] = (to_host(v), to_host(V), to_host(E))
    dham.set_split_format(0)
    e = [rel_err(out[2][i], out[1][i]) for i in range(3)]
    print("fp16 vs tf32 split: vbias %.2e vHS %.2e energy %.2e" % tuple(e))
    assert max(e) < 2e-5
    assert dham.device_error_flag() == 0
