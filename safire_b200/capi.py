"""ctypes binding of the C ABI (include/afqmc_c.h) exported by safire_b200/_lib/libsafire_afqmc.so.

The library is built in-tree (python -m safire_b200.build).  Loading fails loudly when it is
missing: there is no CPU or library fallback behind these functions.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libsafire_afqmc.so")

OK = 0
# status codes of include/afqmc_c.h
(ERR_ARG, ERR_SHAPE, ERR_CUDA, ERR_NONFINITE, ERR_TIMEOUT, ERR_ALLOC, ERR_UNSUPPORTED,
 ERR_COLLAPSE) = range(1, 9)
CLOSED, COLLINEAR = 1, 2
PREC_FP64, PREC_MIXED = 0, 1
STEP_G_READY, STEP_KEEP_G = 1, 2  # afqmc_prop_step_flags
SPLIT_AUTO, SPLIT_TF32, SPLIT_FP16 = 0, 1, 2  # afqmc_ham_set_split_format
(WEIGHT, PHASE, PSEUDO_ELOC, E1, EXX, EJ, OVLP, LOGSCL_UP, LOGSCL_DN, IS_UNITARY,
 THETA) = range(11)
NPROP = 11

vp = C.c_void_p
i32 = C.c_int
i64 = C.c_long
f64 = C.c_double
u64 = C.c_ulonglong


class PropParams(C.Structure):
    _fields_ = [("dt", f64), ("taylor_n", i32), ("vbias_bound", f64),
                ("upper_cutoff_scale", f64), ("lower_cutoff_scale", f64),
                ("weight_bound_floor", f64), ("weight_bound_fraction", f64),
                ("denseP1", i32), ("precision", i32)]


# name: (restype, argtypes)
_SIGS = {
    "afqmc_status_string": (C.c_char_p, [i32]),
    "afqmc_last_error": (C.c_char_p, []),
    "afqmc_version": (i32, []),
    "afqmc_kernel_launches": (u64, []),
    "afqmc_prop_set_timing": (i32, [vp, i32]),
    "afqmc_prop_timings": (i32, [vp, C.POINTER(f64)]),
    "afqmc_log_overlap": (i32, [vp, vp, i64, vp, i32, i32, i32, vp]),
    "afqmc_log_overlap_noalloc": (i32, [vp, vp, i64, vp, i32, i32, i32, vp]),
    "afqmc_mixed_density_matrix": (i32, [vp, vp, i64, vp, i64, vp, i32, i32, i32, i32, vp]),
    "afqmc_mixed_density_matrix_batched": (i32, [vp, i64, vp, i64, vp, i64, vp, i32, i32, i32,
                                                 i32, vp]),
    "afqmc_inverse_logdet": (i32, [vp, vp, vp, i32, i32, vp]),
    "afqmc_orthogonalize": (i32, [vp, i64, vp, i32, i32, i32, vp]),
    "afqmc_propagate": (i32, [vp, vp, vp, i64, i32, i32, i32, i32, vp]),
    "afqmc_ham_create": (i32, [i32, i32, i32, i32, i32, vp, i32, vp, i32, f64, vp, C.POINTER(vp)]),
    "afqmc_ham_create_thc": (i32, [i32, i32, i32, i32, i32, i32, vp, vp, vp, vp, i32, vp, f64,
                                   vp, C.POINTER(vp)]),
    "afqmc_ham_thc_info": (i32, [vp, C.POINTER(i32), C.POINTER(i32)]),
    "afqmc_ham_destroy": (i32, [vp]),
    "afqmc_prop_autotune_tiles": (i32, [vp, vp, C.POINTER(i32), C.POINTER(C.c_float), vp]),
    "afqmc_ham_set_tiles": (i32, [vp, i32, i32]),
    "afqmc_ham_get_tiles": (i32, [vp, C.POINTER(i32), C.POINTER(i32)]),
    "afqmc_ham_info": (i32, [vp, C.POINTER(i32), C.POINTER(i32), C.POINTER(i32), C.POINTER(i32),
                             C.POINTER(i32), C.POINTER(f64)]),
    "afqmc_ham_get_tensors": (i32, [vp, vp, vp, vp]),
    "afqmc_ham_vbias": (i32, [vp, vp, vp, i32, f64, i32, vp]),
    "afqmc_ham_vhs": (i32, [vp, vp, vp, i32, f64, i32, vp]),
    "afqmc_ham_energy": (i32, [vp, vp, vp, i32, i32, i32, i32, i32, vp]),
    "afqmc_ham_one_body_propagator": (i32, [vp, f64, vp, vp]),
    "afqmc_ham_device_error": (i32, [vp, C.POINTER(C.c_uint)]),
    "afqmc_ham_clear_device_error": (i32, [vp]),
    "afqmc_ham_wait_selftest": (i32, [vp, C.c_longlong, vp]),
    "afqmc_ham_set_exchange_split": (i32, [vp, i32]),
    "afqmc_ham_set_vhs_symmetry": (i32, [vp, i32, C.POINTER(i32)]),
    "afqmc_ham_set_split_format": (i32, [vp, i32, C.POINTER(i32)]),
    "afqmc_ham_set_taylor_fused": (i32, [vp, i32]),
    "afqmc_prop_step_flags": (i32, [vp, vp, vp, vp, i32, vp]),
    "afqmc_ph_excited_2body_energy": (i32, [vp, vp, vp, vp, vp, i32, i32, i32, i32, i32, i32,
                                            vp, vp, vp, vp]),
    "afqmc_ph_excited_1body_energy": (i32, [vp, vp, vp, vp, vp, i32, i32, i32, i32, i32, vp, vp]),
    "afqmc_phmsd_create": (i32, [i32, i32, i32, i32, i32, vp, vp, vp, vp, i32, vp, vp, i32, vp,
                                 vp, i32, vp, vp, vp, vp]),
    "afqmc_phmsd_destroy": (i32, [vp]),
    "afqmc_phmsd_log_overlap": (i32, [vp, vp, i64, vp, i32, vp]),
    "afqmc_phmsd_set_hamiltonian": (i32, [vp, vp, i32, vp, i32, i32, C.c_double]),
    "afqmc_phmsd_energy": (i32, [vp, vp, i64, vp, vp, i32, i32, vp]),
    "afqmc_phmsd_density_matrix": (i32, [vp, vp, i64, vp, vp, i32, i32, vp]),
    "afqmc_phmsd_vbias": (i32, [vp, vp, vp, i32, C.c_double, vp]),
    "afqmc_phmsd_info": (i32, [vp, vp]),
    "afqmc_phmsd_set_precision": (i32, [vp, i32]),
    "afqmc_wfn_onerdm": (i32, [vp, vp, vp, i64, vp, vp]),
    "afqmc_prop_autotune": (i32, [vp, vp, vp, vp, vp]),
    "afqmc_ham_set_coulomb_fp64": (i32, [vp, i32]),
    "afqmc_ham_set_mixed_ops": (i32, [vp, i32]),
    "afqmc_nomsd_create": (i32, [i32, vp, vp, C.POINTER(vp)]),
    "afqmc_nomsd_destroy": (i32, [vp]),
    "afqmc_nomsd_log_overlap": (i32, [vp, vp, vp, vp]),
    "afqmc_nomsd_energy": (i32, [vp, vp, vp, vp, i32, vp]),
    "afqmc_nomsd_density_matrix": (i32, [vp, vp, vp, vp, vp]),
    "afqmc_nomsd_vbias": (i32, [vp, vp, vp, i32, C.c_double, vp]),
    "afqmc_prop_set_nomsd": (i32, [vp, vp, vp]),
    "afqmc_phmsd_excitations": (i32, [i32, i32, vp, i32, vp, vp, vp, vp, vp, vp]),
    "afqmc_prop_set_phmsd": (i32, [vp, vp, vp]),
    "afqmc_mlp_create": (i32, [i32, i32, u64, C.POINTER(vp)]),
    "afqmc_mlp_destroy": (i32, [vp]),
    "afqmc_mlp_num_params": (C.c_long, [vp]),
    "afqmc_mlp_set_normalization": (i32, [vp, vp, vp, C.c_float, C.c_float]),
    "afqmc_mlp_params": (i32, [vp, i32, vp, i32]),
    "afqmc_mlp_predict": (i32, [vp, vp, i32, vp, vp]),
    "afqmc_mlp_gradients": (i32, [vp, vp, vp, i32, vp, vp]),
    "afqmc_mlp_train_step": (i32, [vp, vp, vp, i32, C.c_float, vp, vp]),
    "afqmc_exchange_features": (i32, [vp, i64, vp, i64, i32, i32, i32, i32, vp, vp, vp]),
    "afqmc_wset_create": (i32, [i32, i32, i32, i32, i32, C.POINTER(vp)]),
    "afqmc_wset_destroy": (i32, [vp]),
    "afqmc_wset_buffer": (i32, [vp, C.POINTER(vp), C.POINTER(i64), C.POINTER(i32)]),
    "afqmc_wset_get_property": (i32, [vp, i32, vp]),
    "afqmc_wset_set_property": (i32, [vp, i32, vp]),
    "afqmc_wset_init_from_trial": (i32, [vp, vp, vp]),
    "afqmc_wfn_density_matrix": (i32, [vp, vp, vp, vp, vp]),
    "afqmc_wfn_log_overlap": (i32, [vp, vp, vp, vp]),
    "afqmc_wfn_energy": (i32, [vp, vp, vp, vp, i32, i32, vp]),
    "afqmc_wfn_vmf": (i32, [vp, f64, vp]),
    "afqmc_prop_params_default": (None, [C.POINTER(PropParams)]),
    "afqmc_prop_create": (i32, [vp, C.POINTER(PropParams), i32, C.POINTER(vp)]),
    "afqmc_prop_destroy": (i32, [vp]),
    "afqmc_prop_get_p1": (i32, [vp, vp, vp]),
    "afqmc_prop_step": (i32, [vp, vp, f64, vp, vp]),
    "afqmc_prop_step_dev": (i32, [vp, vp, vp, vp, vp]),
    "afqmc_prop_orthogonalize": (i32, [vp, vp, vp]),
    "afqmc_prop_set_field_seed": (i32, [vp, u64]),
    "afqmc_prop_last_step": (i32, [vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp), C.POINTER(vp),
                                   C.POINTER(vp)]),
    "afqmc_prop_bound_stats": (i32, [vp, C.POINTER(C.c_longlong)]),
    "afqmc_split_seed": (u64, [i32, i32, C.c_uint]),
    "afqmc_host_rng_create": (i32, [u64, C.POINTER(vp)]),
    "afqmc_host_rng_destroy": (i32, [vp]),
    "afqmc_host_rng_uniform": (i32, [vp, vp, i64]),
    "afqmc_comb": (i32, [vp, vp, i32, i32, vp]),
    "afqmc_plan_walker_exchange": (i32, [vp, vp, i32, vp, i32, C.POINTER(i32)]),
    "afqmc_population_control": (i32, [vp, vp, vp, vp]),
    "afqmc_wset_copy_rows": (i32, [vp, vp, vp, i32, vp]),
    "afqmc_wset_pack_rows": (i32, [vp, vp, i32, vp, vp]),
    "afqmc_wset_unpack_rows": (i32, [vp, vp, i32, vp, vp]),
    "afqmc_wset_normalize_weights": (i32, [vp, vp]),
    "afqmc_energy_sums": (i32, [vp, vp, vp, vp]),
    "afqmc_pseudo_energy_sums": (i32, [vp, f64, vp, vp]),
}

_lib = None


class AfqmcError(RuntimeError):
    def __init__(self, fn, status, detail):
        super().__init__(f"{fn} failed with status {status}: {detail}")
        self.status = status


def lib():
    """The loaded C-ABI library (raises if the in-tree build is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m safire_b200.build` "
                "(the CUDA path has no fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def call(name, *args):
    """Call an int-returning ABI function and raise AfqmcError on a non-zero status."""
    L = lib()
    st = getattr(L, name)(*args)
    if st != OK:
        raise AfqmcError(name, st, L.afqmc_last_error().decode(errors="replace"))
    return st


def exported_symbols():
    return list(_SIGS)
