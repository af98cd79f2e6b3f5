"""ctypes binding of the C ABI declared in include/safire_b200.h.

Loading fails loudly when the sm_100a library has not been built: there is no CPU fallback.
"""
import ctypes
import os

import numpy as np

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib", "libsafire_b200.so")

SFQ_OK = 0
ERRORS = {1: "SHAPE", 2: "ARG", 3: "UNSUPPORTED", 4: "CUDA", 5: "OOM", 6: "WEIGHT_COLLAPSE", 7: "NONFINITE",
          8: "TIMEOUT", 9: "WORKSPACE", 10: "INTERNAL", 11: "RANK"}
OP_MIXED_DENSITY_MATRIX, OP_LOG_OVERLAP, OP_PROPAGATE, OP_ORTHOGONALIZE, OP_ENERGY, OP_INVERSE_LOGDET = 1, 2, 3, 4, 5, 6

# walker property columns, in the order the engine stores them (WalkerConfig.hpp:28-48 names)
PROPS = ("WEIGHT", "PHASE", "PSEUDO_ELOC_", "E1_", "EXX_", "EJ_", "OVLP", "THETA")
PHASES = ("density", "vbias", "fields", "vHS", "propagate", "overlap", "update", "ortho", "popcontrol", "energy",
          "vHS_gemm", "taylor_gemm")


class SafireError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"SFQ_ERR_{ERRORS.get(code, code)}: {msg}")
        self.code = code


class EngineParams(ctypes.Structure):
    _fields_ = [("nmo", ctypes.c_int), ("nel", ctypes.c_int), ("nchol", ctypes.c_int), ("nwalk", ctypes.c_int),
                ("dt", ctypes.c_double), ("E0", ctypes.c_double), ("taylor_order", ctypes.c_int),
                ("vbias_bound", ctypes.c_double), ("lower_cutoff_scale", ctypes.c_double),
                ("upper_cutoff_scale", ctypes.c_double), ("weight_bound_floor", ctypes.c_double),
                ("weight_bound_fraction", ctypes.c_double), ("subtractMF", ctypes.c_int),
                ("denseP1", ctypes.c_int), ("free_projection", ctypes.c_int),
                ("target_population", ctypes.c_int), ("seed", ctypes.c_ulonglong), ("device", ctypes.c_int),
                ("precision", ctypes.c_int), ("walker_type", ctypes.c_int), ("nel_dn", ctypes.c_int)]

PRECISION_FP64, PRECISION_MIXED, PRECISION_MIXED_FP32, PRECISION_INT8X3, PRECISION_INT8X2 = 0, 1, 2, 3, 4
WALKER_CLOSED, WALKER_COLLINEAR, WALKER_NONCOLLINEAR = 1, 2, 3


class RunParams(ctypes.Structure):
    _fields_ = [("steps", ctypes.c_int), ("walker_ortho_interval", ctypes.c_int),
                ("population_control_interval", ctypes.c_int), ("equilibration_steps", ctypes.c_int),
                ("measure_interval", ctypes.c_int), ("Eshift_relaxation_factor", ctypes.c_double),
                ("step0", ctypes.c_ulonglong), ("steer_eshift", ctypes.c_int)]


class EngineInfo(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in ("SM", "props", "PsiT", "Lnak")] + \
               [("lnak_complex", ctypes.c_int)] + \
               [(n, ctypes.c_void_p) for n in ("Likn", "haj", "v0", "vmf", "P1", "G", "X", "vHS", "hw", "mf",
                                               "new_ovlp")] + \
               [("bound_stats", ctypes.c_ulonglong * 5), ("vhs_packed", ctypes.c_int), ("hcore", ctypes.c_void_p)]


class Tiles(ctypes.Structure):
    _fields_ = [("g_bn", ctypes.c_int), ("vbias_bn", ctypes.c_int), ("vhs_bn", ctypes.c_int),
                ("taylor_half", ctypes.c_int), ("p1_bn", ctypes.c_int), ("vbias_ksplit", ctypes.c_int),
                ("us_builtin", ctypes.c_double * 5), ("us_tuned", ctypes.c_double * 5)]

    PRODUCTS = ("G", "vbias", "vHS", "taylor_term", "P1")

    def choice(self):
        return {k: getattr(self, k) for k in ("g_bn", "vbias_bn", "vhs_bn", "taylor_half", "p1_bn", "vbias_ksplit")}


class ServerParams(ctypes.Structure):
    _fields_ = [("hbm_budget", ctypes.c_size_t), ("max_inflight", ctypes.c_int), ("device", ctypes.c_int)]


class RequestInfo(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("system", ctypes.c_int), ("t_submit", ctypes.c_double),
                ("t_start", ctypes.c_double), ("t_finish", ctypes.c_double), ("Eshift", ctypes.c_double),
                ("nmeas", ctypes.c_int), ("step0", ctypes.c_ulonglong), ("message", ctypes.c_char * 128)]


_lib = None

_VP, _I, _D, _SZ, _U64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_size_t, ctypes.c_ulonglong
_SIGS = {
    "sfq_abi_version": ([], _I),
    "sfq_last_error": ([], ctypes.c_char_p),
    "sfq_memcpy": ([_VP, _VP, _SZ, _I, _VP], _I),
    "sfq_workspace_size": ([_I, _I, _I, _I, _I], _SZ),
    "sfq_mixed_density_matrix": ([_VP, _I, _VP, _VP, _VP, _I, _I, _I, _I, _VP, _SZ, _VP], _I),
    "sfq_log_overlap": ([_VP, _I, _VP, _VP, _I, _I, _I, _VP, _SZ, _VP], _I),
    "sfq_mixed_density_matrix_noalloc": ([_VP, _I, _VP, _VP, _VP, _I, _I, _I, _VP], _I),
    "sfq_noalloc_scratch_bytes": ([], _SZ),
    "sfq_inverse_logdet": ([_VP, _VP, _VP, _I, _I, _VP], _I),
    "sfq_propagate": ([_VP, _VP, _I, _VP, _I, _I, _I, _I, _VP, _SZ, _VP], _I),
    "sfq_orthogonalize": ([_VP, _VP, _I, _I, _I, _VP, _SZ, _VP], _I),
    "sfq_vbias": ([_VP, _VP, _I, _VP, _I, _I, _I, _I, _D, _I, _VP], _I),
    "sfq_vhs": ([_VP, _VP, _VP, _I, _I, _I, _D, _VP], _I),
    "sfq_energy": ([_VP, _VP, _VP, _VP, _I, _D, _I, _I, _I, _I, _I, _I, _I, _VP, _SZ, _VP], _I),
    "sfq_assemble_x": ([_VP, _VP, _VP, _VP, _VP, _U64, _U64, _I, _I, _D, _I, _VP], _I),
    "sfq_comb": ([_VP, _D, _I, _VP, _VP], _I),
    "sfq_comb_host": ([_VP, _D, _I, _I, _VP], _I),
    "sfq_plan_walker_exchange": ([_VP, _VP, _I, _VP, _I, _VP], _I),
    "sfq_walker_moves": ([_VP, _VP, _I, _I, _VP, _I, _VP, _VP, _I, _VP, _VP, _I, _VP], _I),
    "sfq_gemm_split_bf16": ([_VP, _VP, _VP, _I, _I, _I, _I, _I, _I, _I, _I, _VP], _I),
    "sfq_gemm_bf16_planes": ([ctypes.POINTER(_VP), ctypes.POINTER(_VP), _I, _VP, _I, _I, _I, _I, ctypes.c_long,
                              ctypes.c_long, ctypes.c_float, ctypes.c_float, _I, _VP], _I),
    "sfq_split_bf16": ([_VP, ctypes.c_long, _VP, _VP, _VP, _VP], _I),
    "sfq_gemm_int8_slices": ([_VP, _VP, _VP, _I, _I, _I, _I, _I, _I, _VP], _I),
    "sfq_engine_copy_walker": ([_VP, _I, _I], _I),
    "sfq_engine_walker_row_elems": ([_VP], ctypes.c_long),
    "sfq_engine_measure_observables": ([_VP, _VP, _VP, _I, _VP, _VP], _I),
    "sfq_engine_enable_time_evolved_bp": ([_VP], _I),
    "sfq_engine_te_anchor": ([_VP], _I),
    "sfq_engine_te_evolve": ([_VP, _I], _I),
    "sfq_engine_measure_te_rdm": ([_VP, _I, _VP, _VP], _I),
    "sfq_engine_measure_te_observables": ([_VP, _I, _VP, _VP, _I, _VP, _VP], _I),
    "sfq_engine_measure_bp_observables": ([_VP, _I, _I, _I, _VP, _VP, _I, _VP, _VP], _I),
    "sfq_engine_pack_walkers": ([_VP, _VP, _I, _VP], _I),
    "sfq_engine_unpack_walkers": ([_VP, _VP, _I, _VP], _I),
    "sfq_engine_copy_walkers": ([_VP, _VP, _I, _I], _I),
    "sfq_selftest_wait_expiry": ([_U64, _VP], _I),
    "sfq_engine_resize": ([_VP, _I], _I),
    "sfq_one_body_matrix": ([_VP, _VP, _VP, _VP, _I, _I, _D, _VP, _VP], _I),
    "sfq_gemm_int8_cplx_b": ([_VP, _VP, _VP, _I, _I, _I, _I, _I, _VP], _I),
    "sfq_engine_params_default": ([ctypes.POINTER(EngineParams)], None),
    "sfq_engine_create": ([ctypes.POINTER(_VP), ctypes.POINTER(EngineParams), _VP, _VP, _VP], _I),
    "sfq_engine_create_nomsd": ([ctypes.POINTER(_VP), ctypes.POINTER(EngineParams), _VP, _VP, _I, _VP, _VP], _I),
    "sfq_engine_destroy": ([_VP], _I),
    "sfq_engine_synchronize": ([_VP], _I),
    "sfq_engine_stream": ([_VP], _VP),
    "sfq_engine_set_walkers": ([_VP, _VP, _VP], _I),
    "sfq_engine_get_walkers": ([_VP, _VP, _VP], _I),
    "sfq_engine_export_walker_buffer": ([_VP, _VP], _I),
    "sfq_engine_energy": ([_VP, _I, _VP], _I),
    "sfq_engine_propagate": ([_VP, _D, _U64, _VP], _I),
    "sfq_engine_propagate_host": ([_VP, _D, _U64, _VP, _VP], _I),
    "sfq_engine_orthogonalize": ([_VP], _I),
    "sfq_engine_population_control": ([_VP, _U64], _I),
    "sfq_engine_population_control_uniform": ([_VP, ctypes.c_double], _I),
    "sfq_engine_measure_rdm": ([_VP, _VP, _VP], _I),
    "sfq_engine_enable_back_propagation": ([_VP, _I], _I),
    "sfq_engine_bp_anchor": ([_VP], _I),
    "sfq_engine_measure_bp_rdm": ([_VP, _I, _I, _I, _VP, _VP], _I),
    "sfq_engine_averages": ([_VP, ctypes.POINTER(_D), ctypes.POINTER(_D), ctypes.POINTER(_D)], _I),
    "sfq_engine_measure": ([_VP, _VP], _I),
    "sfq_engine_run": ([_VP, ctypes.POINTER(RunParams), ctypes.POINTER(_D), _VP, _I, ctypes.POINTER(_I)], _I),
    "sfq_engine_block": ([_VP, ctypes.POINTER(RunParams), ctypes.POINTER(_D), _VP, _I, ctypes.POINTER(_I)], _I),
    "sfq_engine_block_async": ([_VP, ctypes.POINTER(RunParams), _D], _I),
    "sfq_engine_block_query": ([_VP], _I),
    "sfq_engine_block_result": ([_VP, ctypes.POINTER(_D), _VP, _I, ctypes.POINTER(_I)], _I),
    "sfq_engine_footprint": ([_VP, ctypes.POINTER(_SZ)], _I),
    "sfq_engine_autotune": ([_VP, _I, ctypes.POINTER(Tiles)], _I),
    "sfq_engine_set_tiles": ([_VP, ctypes.POINTER(Tiles)], _I),
    "sfq_engine_tiles": ([_VP, ctypes.POINTER(Tiles)], _I),
    "sfq_group_create": ([ctypes.POINTER(_VP), ctypes.POINTER(_VP), _I], _I),
    "sfq_group_destroy": ([_VP], _I),
    "sfq_group_block": ([_VP, ctypes.POINTER(RunParams), _VP, _VP, _VP, _I, _VP], _I),
    "sfq_group_block_async": ([_VP, ctypes.POINTER(RunParams), _VP], _I),
    "sfq_group_block_query": ([_VP], _I),
    "sfq_group_set_lanes": ([_VP, _I], _I),
    "sfq_group_set_fused": ([_VP, _I], _I),
    "sfq_group_block_result": ([_VP, _VP, _VP, _VP, _I, _VP], _I),
    "sfq_server_create": ([ctypes.POINTER(_VP), ctypes.POINTER(ServerParams)], _I),
    "sfq_server_destroy": ([_VP], _I),
    "sfq_server_add_system": ([_VP, ctypes.POINTER(EngineParams), _VP, _VP, _VP, ctypes.POINTER(_I)], _I),
    "sfq_server_warm": ([_VP, _I], _I),
    "sfq_server_submit": ([_VP, _I, ctypes.POINTER(RunParams), ctypes.POINTER(ctypes.c_longlong)], _I),
    "sfq_server_progress": ([_VP, ctypes.POINTER(_I)], _I),
    "sfq_server_request": ([_VP, ctypes.c_longlong, ctypes.POINTER(RequestInfo), _VP, _I], _I),
    "sfq_server_stats": ([_VP, ctypes.POINTER(_SZ), ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(_I)], _I),
    "sfq_server_clock": ([_VP], _D),
    "sfq_engine_info": ([_VP, ctypes.POINTER(EngineInfo)], _I),
    "sfq_engine_profile": ([_VP, _I], _I),
    "sfq_engine_phase_times": ([_VP, _VP, _VP, _I], _I),
    "sfq_launch_count": ([], ctypes.c_ulonglong),
    "sfq_field_uniforms": ([_VP, _U64, _U64, _I, _I, _VP], _I),
}


def exported_symbols():
    return sorted(_SIGS)


def lib():
    """The loaded library; raises if it was not built (no fallback path exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m safire_b200.build` "
                               "(the AFQMC path has no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (args, res) in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def check(rc):
    if rc != SFQ_OK:
        raise SafireError(rc, lib().sfq_last_error().decode())
    return rc


def ptr(x):
    """Device/host address of a torch tensor or numpy array (None -> NULL)."""
    if x is None:
        return None
    if isinstance(x, np.ndarray):
        return x.ctypes.data
    return x.data_ptr()


def system_params(system, **kw):
    """default_params for a System: CLOSED; COLLINEAR when the system has nel_dn >= 0 down electrons
    (its PsiT then stacks the up rows over the down rows); NONCOLLINEAR when it has npol = 2 (PsiT
    (N, 2M) spinor orbitals)."""
    nel_dn = getattr(system, "nel_dn", -1)
    coll = nel_dn is not None and nel_dn >= 0
    p = default_params(nmo=system.M, nel=system.N - (nel_dn if coll else 0), nchol=system.Nc, **kw)
    if coll:
        p.walker_type, p.nel_dn = WALKER_COLLINEAR, nel_dn
    elif getattr(system, "npol", 1) == 2:
        p.walker_type = WALKER_NONCOLLINEAR
    return p


def default_params(**kw):
    p = EngineParams()
    lib().sfq_engine_params_default(ctypes.byref(p))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p
