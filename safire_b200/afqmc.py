"""Python mirror of the reference's operator API for the walker step, on top of the C ABI.

Names follow bkesk/SAFIRE so that tests and drivers read like the reference's own:

  det_ops.Log_Overlap / MixedDensityMatrix / orthogonalize / Propagate / inverse_logdet
        (src/AFQMC/SlaterDeterminantOperations/*.hpp)
  HamiltonianOperations (Real3IndexFactorization): vbias, vHS, energy,
        getOneBodyPropagatorMatrix, number_of_cholesky_vectors, energy_offset
        (src/AFQMC/HamiltonianOperations/Real3IndexFactorization.hpp)
  NOMSD: MixedDensityMatrix, Log_Overlap, Energy, vMF  (src/AFQMC/Wavefunctions/NOMSD.cpp)
  WalkerSet: getProperty / setProperty / SlaterMatrices  (src/AFQMC/Walkers/WalkerSetBase.h)
  Propagator: Propagate(wset, Eshift), Orthogonalize(wset)  (Propagators/AFQMCBasePropagator.cpp)
  population_control(wset, rng)  (src/AFQMC/Walkers/population_control.hpp)

Device arrays are torch CUDA tensors (complex128 / float64), used only as device memory and
streams; every computation runs in the CUDA library.  Errors raise capi.AfqmcError, the analogue
of the reference's utils::check exceptions.
"""
from __future__ import annotations

import ctypes as C
from types import SimpleNamespace

import numpy as np
import torch

from . import capi
from .capi import call, lib, vp

CLOSED, COLLINEAR = capi.CLOSED, capi.COLLINEAR
PREC_FP64, PREC_MIXED = capi.PREC_FP64, capi.PREC_MIXED


def _stream(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return vp(s.cuda_stream)


def _ptr(t):
    if t is None:
        return None
    if isinstance(t, torch.Tensor):
        if not t.is_cuda and t.numel() > 0:
            raise ValueError("expected a CUDA tensor")
        return vp(t.data_ptr())
    return vp(t)


def _host_ptr(a: np.ndarray):
    return vp(a.ctypes.data)


class _DevView:
    """__cuda_array_interface__ wrapper so torch can view library-owned device memory."""

    def __init__(self, ptr, shape, typestr, strides=None):
        self.__cuda_array_interface__ = dict(shape=tuple(shape), typestr=typestr,
                                             data=(int(ptr), False), version=3,
                                             strides=strides)


def device_view(ptr, shape, dtype=torch.complex128, strides_bytes=None):
    typestr = {torch.complex128: "<c16", torch.float64: "<f8", torch.int32: "<i4"}[dtype]
    return torch.as_tensor(_DevView(ptr, shape, typestr, strides_bytes), device="cuda")


# --------------------------------------------------------------------------------------------
# det_ops
# --------------------------------------------------------------------------------------------
class det_ops:  # noqa: N801 (reference namespace name)
    @staticmethod
    def Log_Overlap(A, B, ovlp, stream=None):
        """A = PsiT [N, M], B = S [W, M, N] (walker stride B.stride(0)), ovlp [W] accumulated."""
        W, M, N = B.shape
        call("afqmc_log_overlap", _ptr(A), _ptr(B), B.stride(0), _ptr(ovlp), W, M, N,
             _stream(stream))

    @staticmethod
    def MixedDensityMatrix(A, B, C_, ovlp, compact=True, stream=None):
        W, M, N = B.shape
        call("afqmc_mixed_density_matrix", _ptr(A), _ptr(B), B.stride(0), _ptr(C_), C_.stride(0),
             _ptr(ovlp), W, M, N, int(bool(compact)), _stream(stream))

    @staticmethod
    def MixedDensityMatrixBatched(A, B, C_, ovlp, compact=True, stream=None):
        """The overload with a bra per walker: A, B [W][M][N] (walker strides A.stride(0),
        B.stride(0)), C_ [W][N][M] (compact) or [W][M][M]."""
        W, M, N = B.shape
        call("afqmc_mixed_density_matrix_batched", _ptr(A), A.stride(0), _ptr(B), B.stride(0),
             _ptr(C_), C_.stride(0), _ptr(ovlp), W, M, N, int(bool(compact)), _stream(stream))

    @staticmethod
    def inverse_logdet(A, Ainv, logdet, stream=None):
        W, N, _ = A.shape
        call("afqmc_inverse_logdet", _ptr(A), _ptr(Ainv), _ptr(logdet), W, N, _stream(stream))

    @staticmethod
    def orthogonalize(A, log_detR, stream=None):
        W, M, N = A.shape
        call("afqmc_orthogonalize", _ptr(A), A.stride(0), _ptr(log_detR), W, M, N,
             _stream(stream))

    @staticmethod
    def Propagate(S, P1, V, order=6, stream=None):
        W, M, N = S.shape
        call("afqmc_propagate", _ptr(P1), _ptr(V), _ptr(S), S.stride(0), W, M, N, order,
             _stream(stream))


# --------------------------------------------------------------------------------------------
# HamiltonianOperations (Real3IndexFactorization)
# --------------------------------------------------------------------------------------------
class HamiltonianOperations:
    def __init__(self, walker_type, M, nup, ndn, Likn, hij, E0, PsiT):
        """Likn float64 [nspin_H2, M, M, Nc]; hij complex [nspin_H1, M, M]; PsiT list of complex
        [N_s, M] (numpy, host)."""
        Likn = np.ascontiguousarray(Likn, dtype=np.float64)
        hij = np.ascontiguousarray(hij, dtype=np.complex128)
        psi = np.ascontiguousarray(np.concatenate([np.asarray(p) for p in PsiT], axis=0),
                                   dtype=np.complex128)
        self.walker_type, self.M, self.nup, self.ndn = walker_type, M, nup, ndn
        self.Nc = Likn.shape[3]
        self.E0 = float(E0)
        self.nel = nup + (ndn if walker_type == COLLINEAR else 0)
        h = vp()
        call("afqmc_ham_create", walker_type, M, nup, ndn, self.Nc, _host_ptr(Likn), Likn.shape[0],
             _host_ptr(hij), hij.shape[0], float(E0), _host_ptr(psi), C.byref(h))
        self.handle = h
        self.nspin_H2 = Likn.shape[0]

    @classmethod
    def thc(cls, walker_type, M, nup, ndn, X, L, hij, E0, PsiT, Z=None, v0=None):
        """THC Hamiltonian operations (THCOps, HamiltonianOperations/THCOps.hpp): X float64
        [M, nu] (Piu), L float64 [nu, nv] (Luv), Z float64 [nu, nu] (rotMuv, default L L^T),
        v0 float64 [M, M] (default from X and Z); the Cholesky vectors this factorisation
        stands for are L_n = X diag(L[:, n]) X^T.  Same methods as the Cholesky form, complex128
        only."""
        X = np.ascontiguousarray(X, dtype=np.float64)
        L = np.ascontiguousarray(L, dtype=np.float64)
        hij = np.ascontiguousarray(hij, dtype=np.complex128)
        Zc = None if Z is None else np.ascontiguousarray(Z, dtype=np.float64)
        v0c = None if v0 is None else np.ascontiguousarray(v0, dtype=np.float64)
        psi = np.ascontiguousarray(np.concatenate([np.asarray(p) for p in PsiT], axis=0),
                                   dtype=np.complex128)
        self = cls.__new__(cls)
        self.walker_type, self.M, self.nup, self.ndn = walker_type, M, nup, ndn
        self.nu, self.Nc = L.shape
        self.E0 = float(E0)
        self.nel = nup + (ndn if walker_type == COLLINEAR else 0)
        h = vp()
        call("afqmc_ham_create_thc", walker_type, M, nup, ndn, self.nu, self.Nc, _host_ptr(X),
             _host_ptr(L), _host_ptr(Zc) if Zc is not None else None, _host_ptr(hij),
             hij.shape[0], _host_ptr(v0c) if v0c is not None else None, float(E0),
             _host_ptr(psi), C.byref(h))
        self.handle = h
        self.nspin_H2 = 1
        return self

    def __del__(self):
        h = getattr(self, "handle", None)
        try:
            if h and capi._lib is not None:
                capi._lib.afqmc_ham_destroy(h)
        except (AttributeError, TypeError):  # interpreter shutdown: the library is gone
            pass
        self.handle = None

    def number_of_cholesky_vectors(self):
        return self.Nc

    def energy_offset(self):
        return self.E0

    def vbias(self, G, v, dt, precision=PREC_FP64, stream=None):
        call("afqmc_ham_vbias", self.handle, _ptr(G), _ptr(v), G.shape[0], float(dt), precision,
             _stream(stream))

    def vHS(self, X, dt, precision=PREC_FP64, stream=None, out=None):
        W = X.shape[0]
        nst = self.nspin_H2 if self.walker_type == COLLINEAR else 1
        V = out if out is not None else torch.empty((nst, W, self.M, self.M),
                                                    dtype=torch.complex128, device=X.device)
        call("afqmc_ham_vhs", self.handle, _ptr(X), _ptr(V), W, float(dt), precision,
             _stream(stream))
        return V

    def energy(self, E, G, addH1=True, addEJ=True, addEXX=True, precision=PREC_FP64,
               stream=None):
        call("afqmc_ham_energy", self.handle, _ptr(G), _ptr(E), G.shape[0], int(addH1),
             int(addEJ), int(addEXX), precision, _stream(stream))

    def getOneBodyPropagatorMatrix(self, dt, vMF):
        nspin = 2 if self.walker_type == COLLINEAR else 1
        vm = np.ascontiguousarray(vMF, dtype=np.complex128)
        H1 = np.zeros((nspin, self.M, self.M), dtype=np.complex128)
        call("afqmc_ham_one_body_propagator", self.handle, float(dt), _host_ptr(vm), _host_ptr(H1))
        return H1

    def set_tiles(self, vbias_bn=128, exchange_block=64):
        """Tile width of the mixed vbias GEMM (128 / 64) and L2 block of the exchange kernel's
        tile order: the results do not depend on them."""
        call("afqmc_ham_set_tiles", self.handle, int(vbias_bn), int(exchange_block))

    def get_tiles(self):
        a, b = C.c_int(), C.c_int()
        call("afqmc_ham_get_tiles", self.handle, C.byref(a), C.byref(b))
        return a.value, b.value

    def set_exchange_split(self, nsplit):
        """3: 3xTF32 exchange contraction (default); 1: plain TF32."""
        call("afqmc_ham_set_exchange_split", self.handle, int(nsplit))

    def set_mixed_ops(self, mask):
        """Mixed precision per operation: 1 vbias, 2 vHS + propagation, 4 energy (default 7)."""
        call("afqmc_ham_set_mixed_ops", self.handle, int(mask))

    def set_coulomb_fp64(self, on=True):
        """Mixed precision: EJ's Coulomb vector from a complex128 GEMM, or (default) from the
        tensor-core exchange traces."""
        call("afqmc_ham_set_coulomb_fp64", self.handle, int(bool(on)))

    def set_vhs_symmetry(self, enable=True):
        """Symmetric mixed-precision vHS (i <= k pairs only) when every Cholesky vector is
        symmetric; returns whether it is in use."""
        active = C.c_int()
        call("afqmc_ham_set_vhs_symmetry", self.handle, int(bool(enable)), C.byref(active))
        return bool(active.value)

    def set_split_format(self, fmt=capi.SPLIT_AUTO):
        """Operand format of the mixed-precision vbias, vHS and exchange (capi.SPLIT_AUTO,
        SPLIT_TF32 or SPLIT_FP16); returns whether the FP16 split runs."""
        active = C.c_int()
        call("afqmc_ham_set_split_format", self.handle, int(fmt), C.byref(active))
        return bool(active.value)

    def set_taylor_fused(self, mode):
        """1/True: one persistent kernel for all Taylor products (default); 0/False: one GEMM
        each; 2 / 3: the persistent kernel with one / two walkers in flight per CTA."""
        call("afqmc_ham_set_taylor_fused", self.handle, int(mode))

    def clear_device_error(self):
        call("afqmc_ham_clear_device_error", self.handle)

    def wait_selftest(self, budget_cycles, stream=None):
        """One bounded device wait that nothing completes (afqmc_ham_wait_selftest); raises
        AfqmcError with status ERR_TIMEOUT when the wait gave up, as it should."""
        call("afqmc_ham_wait_selftest", self.handle, int(budget_cycles), _stream(stream))

    def device_error_flag(self):
        f = C.c_uint()
        call("afqmc_ham_device_error", self.handle, C.byref(f))
        return f.value

    def tensors(self):
        nspin = 2 if self.walker_type == COLLINEAR else 1
        nel = [self.nup, self.ndn if self.walker_type == COLLINEAR else 0]
        Lnak = np.zeros(sum(self.Nc * n * self.M for n in nel[:nspin]), dtype=np.complex128)
        haj = np.zeros((self.nel, self.M), dtype=np.complex128)
        vexx = np.zeros((self.nspin_H2, self.M, self.M), dtype=np.float64)
        call("afqmc_ham_get_tensors", self.handle, _host_ptr(Lnak), _host_ptr(haj),
             _host_ptr(vexx))
        out, off = [], 0
        for s in range(nspin):
            n = self.Nc * nel[s] * self.M
            out.append(Lnak[off:off + n].reshape(self.Nc, nel[s], self.M))
            off += n
        return SimpleNamespace(Lnak=out, haj=haj, vexx=vexx)


Real3IndexFactorization = HamiltonianOperations


# --------------------------------------------------------------------------------------------
# Walker set
# --------------------------------------------------------------------------------------------
class WalkerSet:
    def __init__(self, walker_type, M, nup, ndn, W):
        h = vp()
        call("afqmc_wset_create", walker_type, M, nup, ndn, W, C.byref(h))
        self.handle = h
        self.walker_type, self.M, self.nup, self.W = walker_type, M, nup, W
        self.ndn = ndn if walker_type == COLLINEAR else 0
        data, ws, nw = vp(), C.c_long(), C.c_int()
        call("afqmc_wset_buffer", h, C.byref(data), C.byref(ws), C.byref(nw))
        self.walker_size = ws.value
        self.buffer = device_view(data.value, (W, self.walker_size))
        self.prop0 = M * (self.nup + self.ndn)

    def __del__(self):
        h = getattr(self, "handle", None)
        try:
            if h and capi._lib is not None:
                capi._lib.afqmc_wset_destroy(h)
        except (AttributeError, TypeError):  # interpreter shutdown: the library is gone
            pass
        self.handle = None

    def size(self):
        return self.W

    def SlaterMatrices(self, spin=0):
        """[W, M, N_s] view with the walker stride (WalkerSetBase.h:255-275)."""
        off = 0 if spin == 0 else self.M * self.nup
        n = self.nup if spin == 0 else self.ndn
        return self.buffer[:, off:off + self.M * n].unflatten(1, (self.M, n))

    def getProperty(self, prop):
        out = np.zeros(self.W, dtype=np.complex128)
        call("afqmc_wset_get_property", self.handle, prop, _host_ptr(out))
        return out

    def setProperty(self, prop, values):
        v = np.ascontiguousarray(np.broadcast_to(np.asarray(values, dtype=np.complex128),
                                                 (self.W,)))
        call("afqmc_wset_set_property", self.handle, prop, _host_ptr(v))

    def properties(self):
        return self.buffer[:, self.prop0:self.prop0 + capi.NPROP]

    def init_from_trial(self, ham: HamiltonianOperations, stream=None):
        call("afqmc_wset_init_from_trial", self.handle, ham.handle, _stream(stream))

    def copy_rows(self, dst, src, stream=None):
        """rows dst[j] <- rows src[j] (int32 device tensors)."""
        call("afqmc_wset_copy_rows", self.handle, _ptr(dst), _ptr(src), int(dst.numel()),
             _stream(stream))

    def pack_rows(self, idx, stream=None):
        """[n, walker_size] device tensor holding the rows idx (int32 device tensor)."""
        out = torch.empty((int(idx.numel()), self.walker_size), dtype=torch.complex128,
                          device=self.buffer.device)
        call("afqmc_wset_pack_rows", self.handle, _ptr(idx), int(idx.numel()), _ptr(out),
             _stream(stream))
        return out

    def unpack_rows(self, idx, buf, stream=None):
        """rows idx (int32 device tensor) <- buf [n, walker_size]."""
        call("afqmc_wset_unpack_rows", self.handle, _ptr(idx), int(idx.numel()), _ptr(buf),
             _stream(stream))

    def normalize_weights(self, stream=None):
        """w <- w/|w| for every walker (end of population control)."""
        call("afqmc_wset_normalize_weights", self.handle, _stream(stream))


# --------------------------------------------------------------------------------------------
# NOMSD single-determinant trial
# --------------------------------------------------------------------------------------------
class NOMSD:
    def __init__(self, ham: HamiltonianOperations):
        self.ham = ham

    def MixedDensityMatrix(self, wset: WalkerSet, G=None, ovlp=None, stream=None):
        dev = wset.buffer.device
        G = G if G is not None else torch.empty((wset.W, self.ham.nel * self.ham.M),
                                                dtype=torch.complex128, device=dev)
        ovlp = ovlp if ovlp is not None else torch.empty(wset.W, dtype=torch.complex128,
                                                         device=dev)
        call("afqmc_wfn_density_matrix", self.ham.handle, wset.handle, _ptr(G), _ptr(ovlp),
             _stream(stream))
        return G, ovlp

    def Log_Overlap(self, wset: WalkerSet, ovlp=None, stream=None):
        ovlp = ovlp if ovlp is not None else torch.empty(wset.W, dtype=torch.complex128,
                                                         device=wset.buffer.device)
        call("afqmc_wfn_log_overlap", self.ham.handle, wset.handle, _ptr(ovlp), _stream(stream))
        return ovlp

    def Energy(self, wset: WalkerSet, set_properties=True, precision=PREC_FP64, stream=None):
        dev = wset.buffer.device
        E = torch.empty((wset.W, 3), dtype=torch.complex128, device=dev)
        ov = torch.empty(wset.W, dtype=torch.complex128, device=dev)
        call("afqmc_wfn_energy", self.ham.handle, wset.handle, _ptr(E), _ptr(ov),
             int(set_properties), precision, _stream(stream))
        return E, ov

    def OneRDM(self, wset: WalkerSet, G=None, stream=None):
        """sum_w w_w G_w (full mixed density matrices [nspin][M][M], device) and sum_w w_w."""
        if G is None:
            G, _ = self.MixedDensityMatrix(wset, stream=stream)
        nspin = 2 if self.ham.walker_type == COLLINEAR else 1
        rdm = torch.empty((nspin, self.ham.M, self.ham.M), dtype=torch.complex128,
                          device=G.device)
        call("afqmc_wfn_onerdm", self.ham.handle, wset.handle, _ptr(G), int(G.stride(0)),
             _ptr(rdm), _stream(stream))
        return rdm, wset.properties()[:, capi.WEIGHT].sum()

    def vMF(self, dt):
        v = np.zeros(self.ham.Nc, dtype=np.complex128)
        call("afqmc_wfn_vmf", self.ham.handle, float(dt), _host_ptr(v))
        return v


class NOMSDMulti:
    """NOMSD with several determinants (NOMSD.cpp, ci.size() > 1): one HamiltonianOperations per
    determinant (built with that determinant's PsiT) and the coefficients ci."""

    def __init__(self, hams, ci):
        self.hams = list(hams)
        self.ham = self.hams[0]
        c = np.ascontiguousarray(ci, dtype=np.complex128)
        arr = (vp * len(self.hams))(*[h.handle for h in self.hams])
        h = vp()
        call("afqmc_nomsd_create", len(self.hams), C.cast(arr, vp), _host_ptr(c), C.byref(h))
        self.handle = h
        self.ci = c

    def __del__(self):
        h = getattr(self, "handle", None)
        try:
            if h and capi._lib is not None:
                capi._lib.afqmc_nomsd_destroy(h)
        except (AttributeError, TypeError):  # interpreter shutdown: the library is gone
            pass
        self.handle = None

    def Log_Overlap(self, wset: WalkerSet, ovlp=None, stream=None):
        ovlp = ovlp if ovlp is not None else torch.empty(wset.W, dtype=torch.complex128,
                                                         device=wset.buffer.device)
        call("afqmc_nomsd_log_overlap", self.handle, wset.handle, _ptr(ovlp), _stream(stream))
        return ovlp

    def Energy(self, wset: WalkerSet, set_properties=True, precision=PREC_FP64, stream=None):
        dev = wset.buffer.device
        E = torch.empty((wset.W, 3), dtype=torch.complex128, device=dev)
        ov = torch.empty(wset.W, dtype=torch.complex128, device=dev)
        call("afqmc_nomsd_energy", self.handle, wset.handle, _ptr(E), _ptr(ov), precision,
             _stream(stream))
        if set_properties:
            p = wset.properties()
            p[:, capi.OVLP] = ov
            p[:, capi.E1], p[:, capi.EXX], p[:, capi.EJ] = E[:, 0], E[:, 1], E[:, 2]
        return E, ov

    def MixedDensityMatrix(self, wset: WalkerSet, stream=None):
        """(G [W, nspin, M, M] full, ovlp [W]) as NOMSD::MixedDensityMatrix returns them."""
        nspin = 2 if self.ham.walker_type == COLLINEAR else 1
        dev = wset.buffer.device
        G = torch.empty((wset.W, nspin, self.ham.M, self.ham.M), dtype=torch.complex128,
                        device=dev)
        ov = torch.empty(wset.W, dtype=torch.complex128, device=dev)
        call("afqmc_nomsd_density_matrix", self.handle, wset.handle, _ptr(G), _ptr(ov),
             _stream(stream))
        return G, ov

    def vbias(self, G, v, dt, stream=None):
        call("afqmc_nomsd_vbias", self.handle, _ptr(G), _ptr(v), int(G.shape[0]), float(dt),
             _stream(stream))
        return v


class PHMSDWavefunction:
    """The walker-set facade of a PHMSD trial (Wavefunction.hpp's variant over PHMSD.hpp): the
    same calls as NOMSD, evaluated by the multi-determinant kernels.  Energy(precision=PREC_MIXED)
    evaluates the excited determinants' 2-body terms in complex64 (afqmc_phmsd_set_precision)."""

    def __init__(self, trial: "PHMSD", block=0):
        self.ph = trial
        self.block = block
        self.M, self.nup, self.ndn, na_up, na_dn, self.Nc = trial.info()
        self.nact = na_up + na_dn

    def MixedDensityMatrix(self, wset: WalkerSet, G=None, ovlp=None, stream=None):
        dev = wset.buffer.device
        G = G if G is not None else torch.empty((wset.W, self.nact, self.M),
                                                dtype=torch.complex128, device=dev)
        ovlp = ovlp if ovlp is not None else torch.empty(wset.W, dtype=torch.complex128,
                                                         device=dev)
        self.ph.MixedDensityMatrix(wset.buffer, G, ovlp, self.block, stream)
        return G, ovlp

    def Log_Overlap(self, wset: WalkerSet, ovlp=None, stream=None):
        ovlp = ovlp if ovlp is not None else torch.empty(wset.W, dtype=torch.complex128,
                                                         device=wset.buffer.device)
        self.ph.Log_Overlap(wset.buffer, ovlp, stream)
        return ovlp

    def Energy(self, wset: WalkerSet, set_properties=True, precision=PREC_FP64, stream=None):
        dev = wset.buffer.device
        E = torch.empty((wset.W, 3), dtype=torch.complex128, device=dev)
        ov = torch.empty(wset.W, dtype=torch.complex128, device=dev)
        self.ph.set_precision(precision)
        self.ph.Energy(wset.buffer, E, ov, self.block, stream)
        if set_properties:  # PHMSD::Energy(wset) (PHMSD.cpp:75-87)
            p = wset.properties()
            p[:, capi.OVLP] = ov
            p[:, capi.E1], p[:, capi.EXX], p[:, capi.EJ] = E[:, 0], E[:, 1], E[:, 2]
        return E, ov


# --------------------------------------------------------------------------------------------
# Propagator
# --------------------------------------------------------------------------------------------
def default_params(**kw):
    p = capi.PropParams()
    lib().afqmc_prop_params_default(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


class Propagator:
    def __init__(self, ham: HamiltonianOperations, params: capi.PropParams, max_walkers):
        h = vp()
        call("afqmc_prop_create", ham.handle, C.byref(params), int(max_walkers), C.byref(h))
        self.handle = h
        self.ham = ham
        self.params = params

    def __del__(self):
        h = getattr(self, "handle", None)
        try:
            if h and capi._lib is not None:
                capi._lib.afqmc_prop_destroy(h)
        except (AttributeError, TypeError):  # interpreter shutdown: the library is gone
            pass
        self.handle = None

    def P1_vMF(self):
        nspin = 2 if self.ham.walker_type == COLLINEAR else 1
        P1 = np.zeros((nspin, self.ham.M, self.ham.M), dtype=np.complex128)
        vMF = np.zeros(self.ham.Nc, dtype=np.complex128)
        call("afqmc_prop_get_p1", self.handle, _host_ptr(P1), _host_ptr(vMF))
        return P1, vMF

    def set_field_seed(self, seed):
        call("afqmc_prop_set_field_seed", self.handle, int(seed))

    def autotune(self, wset: WalkerSet, stream=None):
        """Picks the fastest Taylor propagation variant for these walkers (mixed precision);
        returns (mode or -1, {mode: step ms}).  The walkers are left as they were."""
        best = C.c_int()
        ms = np.zeros(7, dtype=np.float32)
        call("afqmc_prop_autotune", self.handle, wset.handle, C.byref(best), _host_ptr(ms),
             _stream(stream))
        return best.value, {m: float(t) for m, t in zip((0, 2, 3, 4, 5, 6, 7), ms) if t > 0}

    def autotune_tiles(self, wset: WalkerSet, stream=None):
        """Picks the tile shapes / orders that leave the results bit for bit the same (vbias
        tile width, vHS form, exchange L2 block) on these walkers; returns ({'vbias_bn',
        'vhs_symmetric', 'exchange_block'}, {candidate: ms}).  The walkers are left as they
        were."""
        ch = (C.c_int * 3)()
        ms = np.zeros(8, dtype=np.float32)
        call("afqmc_prop_autotune_tiles", self.handle, wset.handle, ch,
             ms.ctypes.data_as(C.POINTER(C.c_float)), _stream(stream))
        names = ["vbias_bn=128", "vbias_bn=64", "vhs_symmetric", "vhs_all_pairs",
                 "exchange_block=16", "exchange_block=32", "exchange_block=64",
                 "exchange_block=128"]
        return ({"vbias_bn": ch[0], "vhs_symmetric": ch[1], "exchange_block": ch[2]},
                {n: float(t) for n, t in zip(names, ms) if t > 0})

    def set_trial(self, trial, vMF=None):
        """Steps with a multi-determinant trial (PHMSD or NOMSDMulti: vbias and overlaps from
        it); vMF host [Nc] or None keeps the current mean field.  trial None detaches."""
        v = None if vMF is None else np.ascontiguousarray(vMF, dtype=np.complex128)
        vp_ = None if v is None else _host_ptr(v)
        if trial is None:
            prev = getattr(self, "_trial", None)
            name = "afqmc_prop_set_nomsd" if isinstance(prev, NOMSDMulti) else \
                "afqmc_prop_set_phmsd"
            call(name, self.handle, None, vp_)
        elif isinstance(trial, NOMSDMulti):
            call("afqmc_prop_set_nomsd", self.handle, trial.handle, vp_)
        else:
            call("afqmc_prop_set_phmsd", self.handle, trial.handle, vp_)
        self._trial = trial  # the trial must outlive the propagator's use of it

    def Propagate(self, wset: WalkerSet, Eshift, uniforms=None, stream=None):
        """One step.  uniforms: device float64 [W, Nc] or None (device Philox generator)."""
        call("afqmc_prop_step", self.handle, wset.handle, float(Eshift), _ptr(uniforms),
             _stream(stream))

    def Propagate_dev(self, wset: WalkerSet, Eshift_dev, uniforms=None, stream=None):
        call("afqmc_prop_step_dev", self.handle, wset.handle, _ptr(Eshift_dev), _ptr(uniforms),
             _stream(stream))

    def Propagate_flags(self, wset: WalkerSet, Eshift_dev, uniforms=None, flags=0, stream=None):
        """One step with explicit density-matrix reuse (capi.STEP_G_READY / STEP_KEEP_G)."""
        call("afqmc_prop_step_flags", self.handle, wset.handle, _ptr(Eshift_dev), _ptr(uniforms),
             int(flags), _stream(stream))

    def Orthogonalize(self, wset: WalkerSet, stream=None):
        call("afqmc_prop_orthogonalize", self.handle, wset.handle, _stream(stream))

    def last_step(self, W):
        ptrs = [vp() for _ in range(5)]
        call("afqmc_prop_last_step", self.handle, *[C.byref(p) for p in ptrs])
        Nc = self.ham.Nc
        vb, X, hw, mf, nov = (p.value for p in ptrs)
        return SimpleNamespace(vbias=device_view(vb, (W, Nc)), X=device_view(X, (W, Nc)),
                               HW=device_view(hw, (W,)), mf=device_view(mf, (W,)),
                               new_ovlp=device_view(nov, (W,)))

    PHASES = ("G_for_vbias", "vbias", "assemble_X", "vHS", "propagate", "pseudo_energy", "extra")

    def set_timing(self, enable=True):
        call("afqmc_prop_set_timing", self.handle, int(enable))

    def timings(self):
        ms = (C.c_double * len(self.PHASES))()
        call("afqmc_prop_timings", self.handle, ms)
        return dict(zip(self.PHASES, list(ms)))

    def bound_stats(self):
        c = (C.c_longlong * 6)()
        call("afqmc_prop_bound_stats", self.handle, c)
        return list(c)


# --------------------------------------------------------------------------------------------
# population control and estimators
# --------------------------------------------------------------------------------------------
def split_seed(seed, rank, stream):
    return int(lib().afqmc_split_seed(seed, rank, stream))


class HostRandomGenerator:
    """std::mt19937 + uniform_real_distribution<double> (src/utilities/Random.hpp:37-51)."""

    def __init__(self, seed64):
        h = vp()
        call("afqmc_host_rng_create", int(seed64), C.byref(h))
        self.handle = h

    def __del__(self):
        h = getattr(self, "handle", None)
        try:
            if h and capi._lib is not None:
                capi._lib.afqmc_host_rng_destroy(h)
        except (AttributeError, TypeError):  # interpreter shutdown: the library is gone
            pass
        self.handle = None

    def sample_uniform(self, n):
        out = np.empty(n, dtype=np.float64)
        call("afqmc_host_rng_uniform", self.handle, _host_ptr(out), int(n))
        return out


def comb(rng: HostRandomGenerator, weights, num_target):
    w = np.ascontiguousarray(weights, dtype=np.float64)
    off = np.zeros(w.size, dtype=np.int32)
    call("afqmc_comb", rng.handle, _host_ptr(w), w.size, int(num_target), _host_ptr(off))
    return off


def plan_walker_exchange(offspring, counts):
    off = np.ascontiguousarray(offspring, dtype=np.int32)
    cnt = np.ascontiguousarray(counts, dtype=np.int32)
    n = C.c_int()
    call("afqmc_plan_walker_exchange", _host_ptr(off), _host_ptr(cnt), cnt.size, None, 0,
         C.byref(n))
    plan = np.zeros((max(n.value, 1), 4), dtype=np.int32)
    call("afqmc_plan_walker_exchange", _host_ptr(off), _host_ptr(cnt), cnt.size, _host_ptr(plan),
         n.value, C.byref(n))
    return [tuple(int(x) for x in r) for r in plan[:n.value]]


def population_control(wset: WalkerSet, rng: HostRandomGenerator, stream=None):
    off = np.zeros(wset.W, dtype=np.int32)
    call("afqmc_population_control", wset.handle, rng.handle, _host_ptr(off), _stream(stream))
    return off


def energy_sums(wset: WalkerSet, E, out=None, stream=None):
    out = out if out is not None else torch.empty(4, dtype=torch.complex128,
                                                  device=wset.buffer.device)
    call("afqmc_energy_sums", wset.handle, _ptr(E), _ptr(out), _stream(stream))
    return out


def pseudo_energy_sums(wset: WalkerSet, dt, out=None, stream=None):
    out = out if out is not None else torch.empty(2, dtype=torch.complex128,
                                                  device=wset.buffer.device)
    call("afqmc_pseudo_energy_sums", wset.handle, float(dt), _ptr(out), _stream(stream))
    return out


# --------------------------------------------------------------------------------------------
# PHMSD energy kernels (Wavefunctions/detail/phmsd_impl.hpp)
# --------------------------------------------------------------------------------------------
class phmsd:  # noqa: N801 (reference namespace of the free functions)
    @staticmethod
    def ph_excited_2body_energy(iexcit, refc, Twina, R, wgt, EX, EJ, KE, stream=None):
        """EX -= 1/2 wgt eX, EJ += 1/2 wgt (K.K - eJ0), KE written (device tensors; iexcit
        [ndet][2*nex] int32, refc [nelec] int32, Twina [nw][nelec][nchol][nact],
        R [nw][ndet][nex][nact], wgt [ndet][nw])."""
        nw, ndet, nex, nact = R.shape
        nelec, nchol = Twina.shape[1], Twina.shape[2]
        call("afqmc_ph_excited_2body_energy", _ptr(iexcit), _ptr(refc), _ptr(Twina), _ptr(R),
             _ptr(wgt), nw, ndet, nex, nact, nelec, nchol, _ptr(EX), _ptr(EJ), _ptr(KE),
             _stream(stream))

    @staticmethod
    def ph_excited_1body_energy(iexcit, refc, S, R, wgt, E, stream=None):
        """E += sum_d wgt sum_p (S.R + S[particle] - S[refc]) (device tensors; S [nw][nelec][nact])."""
        nw, ndet, nex, nact = R.shape
        nelec = S.shape[1]
        call("afqmc_ph_excited_1body_energy", _ptr(iexcit), _ptr(refc), _ptr(S), _ptr(R),
             _ptr(wgt), nw, ndet, nex, nact, nelec, _ptr(E), _stream(stream))


class PHMSD:
    """Particle-hole multi-determinant trial (Wavefunctions/PHMSD.hpp) from a
    safire_b200.synth.PHMSDTrial (or any object with the same fields)."""

    def __init__(self, trial):
        self.trial = trial
        arrs = []

        def keep(a, dtype):
            a = np.ascontiguousarray(a, dtype=dtype)
            arrs.append(a)
            return _host_ptr(a)

        nu, ne, ex = [], [], []
        for s in (0, 1):
            n_list, e_list = [], []
            for n in sorted(trial.exc[s]):
                for e in trial.exc[s][n]:
                    n_list.append(n)
                    e_list.extend(int(x) for x in e)
            nu.append(1 + len(n_list))
            ne.append(np.array(n_list or [0], dtype=np.int32))
            ex.append(np.array(e_list or [0], dtype=np.int32))
        self.nuniq = nu
        h = vp()
        call("afqmc_phmsd_create", trial.M, trial.nup, trial.ndn, trial.orbmat[0].shape[0],
             trial.orbmat[1].shape[0], keep(trial.orbmat[0], np.complex128),
             keep(trial.orbmat[1], np.complex128), keep(trial.refc[0], np.int32),
             keep(trial.refc[1], np.int32), nu[0], keep(ne[0], np.int32), keep(ex[0], np.int32),
             nu[1], keep(ne[1], np.int32), keep(ex[1], np.int32), int(trial.coef.size),
             keep(trial.det_up, np.int32), keep(trial.det_dn, np.int32),
             keep(trial.coef, np.complex128), C.byref(h))
        self.handle = h

    def __del__(self):
        h = getattr(self, "handle", None)
        try:
            if h and capi._lib is not None:
                capi._lib.afqmc_phmsd_destroy(h)
        except (AttributeError, TypeError):  # interpreter shutdown: the library is gone
            pass
        self.handle = None

    def set_hamiltonian(self, Likn, hij, E0):
        """Likn real [nspin_H2, M, M, Nc], hij complex [nspin_H1, M, M] (host)."""
        L = np.ascontiguousarray(Likn, dtype=np.float64)
        h = np.ascontiguousarray(hij, dtype=np.complex128)
        call("afqmc_phmsd_set_hamiltonian", self.handle, _host_ptr(L), L.shape[0], _host_ptr(h),
             h.shape[0], L.shape[3], float(E0))

    def Energy(self, wbuf, E, ovlp, block=0, stream=None):
        """E [W, 3] (device) and ovlp [W] (device) of every walker row of wbuf [W][ldS]."""
        call("afqmc_phmsd_energy", self.handle, _ptr(wbuf), int(wbuf.stride(0)), _ptr(E),
             _ptr(ovlp), int(wbuf.shape[0]), int(block), _stream(stream))

    def Log_Overlap(self, wbuf, ovlp, stream=None):
        """ovlp [W] (device) <- log overlap of every walker row of wbuf [W][ldS] (device)."""
        call("afqmc_phmsd_log_overlap", self.handle, _ptr(wbuf), int(wbuf.stride(0)), _ptr(ovlp),
             int(wbuf.shape[0]), _stream(stream))

    def set_precision(self, precision):
        """PREC_MIXED: the energy's excited-determinant tables in complex64 (afqmc_phmsd_set_precision)."""
        call("afqmc_phmsd_set_precision", self.handle, int(precision))

    def info(self):
        """(M, nup, ndn, nact_up, nact_dn, Nc)"""
        d = np.zeros(6, dtype=np.int32)
        call("afqmc_phmsd_info", self.handle, _host_ptr(d))
        return tuple(int(x) for x in d)

    def MixedDensityMatrix(self, wbuf, G, ovlp, block=0, stream=None):
        """G [W, nact_up + nact_dn, M] (device) and ovlp [W] (device) of every walker row."""
        call("afqmc_phmsd_density_matrix", self.handle, _ptr(wbuf), int(wbuf.stride(0)), _ptr(G),
             _ptr(ovlp), int(wbuf.shape[0]), int(block), _stream(stream))

    def vbias(self, G, v, dt, stream=None):
        """v [W, Nc] (device) <- sqrt(dt) sum_s Lnak_s . G_s (G from MixedDensityMatrix)."""
        call("afqmc_phmsd_vbias", self.handle, _ptr(G), _ptr(v), int(G.shape[0]), float(dt),
             _stream(stream))
