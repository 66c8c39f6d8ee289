"""ctypes binding of the native library ``libripples_b200.so`` (C ABI in
``include/ripples_b200.h``).

The library is built in-tree by :mod:`ripples_b200.build`.  There is no
fallback: if the shared object is missing or fails to load, importing the
package raises, and every compute entry point reports CUDA errors as
exceptions instead of silently doing something else.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libripples_b200.so")

OK = 0
ERR = {
    -1: "invalid argument",
    -2: "CUDA error",
    -3: "out of device memory / budget",
    -4: "invalid state",
    -5: "size limit exceeded",
    -6: "device-reported error",
}

MODEL_IC, MODEL_LT = 0, 1
DIST_UNIFORM, DIST_NORMAL, DIST_CONST = 0, 1, 2
TIE_REF_HEAP, TIE_LOWEST_ID = 0, 1
SAMPLER_AUTO, SAMPLER_PLAIN, SAMPLER_FUSED = 0, 1, 2
WEIGHTS_UNIFORM, WEIGHTS_LT_NORMALIZED, WEIGHTS_WC = 0, 1, 2
MAX_ROUNDS = 64


class RipError(RuntimeError):
    def __init__(self, code: int, where: str, detail: str = ""):
        self.code = code
        msg = f"{where}: {ERR.get(code, 'error')} ({code})"
        if detail:
            msg += f": {detail}"
        super().__init__(msg)


class ImmRecord(ctypes.Structure):
    _fields_ = [
        ("theta", ctypes.c_uint64),
        ("num_rounds", ctypes.c_uint32),
        ("theta_prime_deltas", ctypes.c_uint64 * MAX_ROUNDS),
        ("round_generate_ms", ctypes.c_double * MAX_ROUNDS),
        ("round_select_ms", ctypes.c_double * MAX_ROUNDS),
        ("theta_estimation_ms", ctypes.c_double),
        ("generate_ms", ctypes.c_double),
        ("select_ms", ctypes.c_double),
        ("total_ms", ctypes.c_double),
        ("f", ctypes.c_double),
        ("total_sets", ctypes.c_uint64),
        ("pool_elements", ctypes.c_uint64),
        ("rrr_set_bytes", ctypes.c_uint64),
    ]


class TsvOptions(ctypes.Structure):
    _fields_ = [
        ("weighted", ctypes.c_int),
        ("undirected", ctypes.c_int),
        ("renumber", ctypes.c_int),
        ("model", ctypes.c_int),
        ("distribution", ctypes.c_int),
        ("mean", ctypes.c_double),
        ("variance", ctypes.c_double),
        ("scale", ctypes.c_double),
    ]


class OpimcRecord(ctypes.Structure):
    _fields_ = [
        ("theta_zero", ctypes.c_uint64),
        ("theta_max", ctypes.c_uint64),
        ("theta", ctypes.c_uint64),
        ("rounds", ctypes.c_uint32),
        ("coverage1", ctypes.c_uint64),
        ("coverage2", ctypes.c_uint64),
        ("lower", ctypes.c_float),
        ("upper", ctypes.c_float),
        ("total_ms", ctypes.c_double),
    ]


class ImmQuery(ctypes.Structure):
    _fields_ = [
        ("graph", ctypes.c_void_p),
        ("k", ctypes.c_uint32),
        ("epsilon", ctypes.c_double),
        ("l", ctypes.c_double),
        ("seed", ctypes.c_uint64),
        ("tiebreak", ctypes.c_int),
        ("seeds", ctypes.c_void_p),
        ("num_seeds", ctypes.c_uint32),
        ("status", ctypes.c_int),
        ("done", ctypes.c_int),
        ("f", ctypes.c_double),
        ("queue_ms", ctypes.c_double),
        ("latency_ms", ctypes.c_double),
        ("record", ImmRecord),
    ]


P = ctypes.c_void_p
U32, U64, I32, I64, DBL, SZ = (ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int,
                               ctypes.c_int64, ctypes.c_double, ctypes.c_size_t)
PP = ctypes.POINTER(ctypes.c_void_p)

# name -> (restype, argtypes); every symbol of include/ripples_b200.h
SIGNATURES = {
    "rip_version": (ctypes.c_char_p, []),
    "rip_ctx_create": (I32, [I32, SZ, PP]),
    "rip_ctx_destroy": (I32, [P]),
    "rip_last_error": (ctypes.c_char_p, [P]),
    "rip_sync": (I32, [P]),
    "rip_ctx_memory": (I32, [P, ctypes.POINTER(SZ), ctypes.POINTER(SZ)]),
    "rip_ctx_stream": (I32, [P, PP]),
    "rip_kernel_launches": (U64, []),
    "rip_graph_uniform_thresholds": (I32, [P, I32, ctypes.POINTER(I32)]),
    "rip_graph_branching": (I32, [P, ctypes.POINTER(ctypes.c_double)]),
    "rip_graph_from_edges": (I32, [P, P, P, P, U64, I32, I32, PP]),
    "rip_graph_id_map": (I32, [P, P]),
    "rip_coin_rate": (I32, [P, ctypes.POINTER(ctypes.c_double)]),
    "rip_graph_upload": (I32, [P, P, P, P, U32, U64, I32, PP]),
    "rip_graph_destroy": (I32, [P]),
    "rip_graph_info": (I32, [P, ctypes.POINTER(U32), ctypes.POINTER(U64), ctypes.POINTER(I32)]),
    "rip_graph_thresholds": (I32, [P, P]),
    "rip_graph_export": (I32, [P, P, P]),
    "rip_rmat_keys_device": (I32, [P, U32, U64, U64, DBL, DBL, DBL, U64, P]),
    "rip_er_keys_device": (I32, [P, U32, U64, U64, U64, P]),
    "rip_graph_from_keys": (I32, [P, P, U64, U32, I32, U64, DBL, DBL, I32, PP]),
    "rip_pool_create": (I32, [P, P, PP]),
    "rip_pool_destroy": (I32, [P]),
    "rip_pool_clear": (I32, [P]),
    "rip_pool_info": (I32, [P, ctypes.POINTER(U64), ctypes.POINTER(U64)]),
    "rip_sample": (I32, [P, U64, U64, I32]),
    "rip_pool_export": (I32, [P, U64, U64, P, P]),
    "rip_pool_import": (I32, [P, P, P, U64]),
    "rip_pool_stats": (I32, [P, P]),
    "rip_pool_timing": (I32, [P, ctypes.POINTER(DBL), ctypes.POINTER(U64), ctypes.POINTER(DBL)]),
    "rip_pool_configure": (I32, [P, U32, U32, U32]),
    "rip_pool_work_caps": (I32, [P, U64, U64]),
    "rip_pool_select_guess": (I32, [P, U32]),
    "rip_pool_heavy_batch": (I32, [P, U32]),
    "rip_pool_heavy_block": (I32, [P, U32]),
    "rip_pool_plain_occupancy": (I32, [P, I32]),
    "rip_graph_autotune": (I32, [P, U64, U32, P, ctypes.POINTER(I32)]),
    "rip_select": (I32, [P, U64, U32, I32, P, P, ctypes.POINTER(U32), ctypes.POINTER(DBL)]),
    "rip_select_counts": (I32, [P, P]),
    "rip_selftest_heap": (I32, [U64, U32, U64]),
    "rip_selftest_heap_device": (I32, [P, U64, U32, U64]),
    "rip_select_profile": (I32, [P, P]),
    "rip_count": (I32, [P, U64, P]),
    "rip_pool_skip": (I32, [P, U64]),
    "rip_shard_begin": (I32, [P, U64, P, ctypes.POINTER(U64)]),
    "rip_shard_pick": (I32, [P, P, ctypes.POINTER(U32), ctypes.POINTER(U64)]),
    "rip_shard_cover": (I32, [P, U32, U64, P]),
    "rip_shard_cover_list": (I32, [P, U32, U64, P, U64, ctypes.POINTER(U64)]),
    "rip_shard_apply": (I32, [P, P, P, U64]),
    "rip_imm": (I32, [P, P, U32, DBL, DBL, U64, I32, I32, P, ctypes.POINTER(U32),
                      ctypes.POINTER(ImmRecord)]),
    "rip_imm_pool": (I32, [P, U32, DBL, DBL, U64, I32, I32, P, ctypes.POINTER(U32),
                           ctypes.POINTER(ImmRecord)]),
    "rip_sample_multi": (I32, [P, P, P, P, U32]),
    "rip_spread_ic": (I32, [P, P, U32, U64, U64, P, P, ctypes.POINTER(ctypes.c_double)]),
    "rip_spread_lt": (I32, [P, P, P, U32, U64, U64, P, P, ctypes.POINTER(ctypes.c_double)]),
    "rip_imm_batch": (I32, [P, ctypes.POINTER(ImmQuery), U32]),
    "rip_server_create": (I32, [P, SZ, U32, PP]),
    "rip_server_destroy": (I32, [P]),
    "rip_server_submit": (I32, [P, ctypes.POINTER(ImmQuery)]),
    "rip_server_tick": (I32, [P, ctypes.POINTER(U32)]),
    "rip_server_pending": (I32, [P, ctypes.POINTER(U32), ctypes.POINTER(U32)]),
    "rip_server_stats": (I32, [P, P]),
    "rip_sample_static": (I32, [P, P, U32, U64, I32, U64, U64, U32, P, U64, P, P,
                                ctypes.POINTER(U64), P]),
    "rip_static_last_error": (ctypes.c_char_p, []),
    "rip_theta_prime": (I64, [I64, DBL, DBL, U64, U64]),
    "rip_inv_theta_prime": (I64, [I64, DBL, DBL, U64, U64]),
    "rip_theta": (U64, [DBL, DBL, U64, DBL, U64]),
    "rip_log_binomial": (DBL, [U64, U64]),
    "rip_rmat_csr": (I32, [U32, U64, DBL, DBL, DBL, U64, PP, PP, ctypes.POINTER(U64)]),
    "rip_er_csr": (I32, [U32, U64, U64, PP, PP, ctypes.POINTER(U64)]),
    "rip_make_weights": (I32, [I32, U32, P, U64, U64, DBL, DBL, P]),
    "rip_write_binary": (I32, [ctypes.c_char_p, U32, U64, P, P, P, I32]),
    "rip_free": (None, [P]),
    "rip_read_tsv_edges": (I32, [ctypes.c_char_p, ctypes.POINTER(TsvOptions),
                                 ctypes.POINTER(U64), P, P, P]),
    "rip_read_tsv": (I32, [ctypes.c_char_p, ctypes.POINTER(TsvOptions), ctypes.POINTER(U32),
                           ctypes.POINTER(U64), P, P, P, P]),
    "rip_read_binary": (I32, [ctypes.c_char_p, ctypes.c_double, ctypes.POINTER(U32),
                              ctypes.POINTER(U64), P, P, P, P]),
    "rip_read_error": (ctypes.c_char_p, []),
    "rip_read_binary_forward": (I32, [ctypes.c_char_p, ctypes.c_double, ctypes.POINTER(U32),
                                      ctypes.POINTER(U64), P, P, P, P]),
    "rip_transpose_csr": (I32, [U32, U64, P, P, P, P, P, P]),
    "rip_coverage": (I32, [P, U64, P, U32, ctypes.POINTER(U64)]),
    "rip_opimc_pool": (I32, [P, P, U32, ctypes.c_float, ctypes.c_float, U64, I32, I32, P,
                             ctypes.POINTER(U32), ctypes.POINTER(OpimcRecord)]),
    "rip_opimc_theta_max": (U64, [U64, ctypes.c_float, U64, ctypes.c_float]),
    "rip_opimc_theta_zero": (U64, [U64, ctypes.c_float, U64, ctypes.c_float]),
    "rip_opimc_lower_bound": (ctypes.c_float, [U64, ctypes.c_float, U64, U64]),
    "rip_opimc_upper_bound": (ctypes.c_float, [U64, ctypes.c_float, U64, U64]),
}


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    if not os.path.exists(path):
        raise ImportError(
            f"native library not found at {path}; build it with "
            "`python ripples_b200/build.py` (the package has no non-CUDA fallback)")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = load()


def check(rc: int, where: str, ctx=None) -> None:
    if rc != OK:
        detail = ""
        if ctx is not None:
            d = lib.rip_last_error(ctx)
            detail = d.decode() if d else ""
        raise RipError(rc, where, detail)
