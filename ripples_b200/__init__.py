"""ripples_b200 -- B200-native (sm_100a) IMM hot path of pnnl/ripples.

RRR-set sampling (IC fused multi-colour BFS / one set per warp, LT walk) and
greedy max-coverage seed selection on the GPU, behind a C ABI
(``include/ripples_b200.h``) and a reference-shaped host API (:mod:`.imm`).
"""
from . import _lib
from ._lib import (MODEL_IC, MODEL_LT, SAMPLER_AUTO, SAMPLER_FUSED, SAMPLER_PLAIN,
                   TIE_LOWEST_ID, TIE_REF_HEAP, WEIGHTS_LT_NORMALIZED, WEIGHTS_UNIFORM,
                   WEIGHTS_WC, RipError)
from .graph import (Context, DeviceGraph, HostGraph, Pool, Query, Server, imm_batch, sample_multi,
                    opimc, spread_ic, spread_lt)
from .imm import (B200RRRGenerator, FindMostInfluentialSet, GenerateRRRSets, IMM,
                  IMMConfiguration, IMMExecutionRecord, independent_cascade_tag,
                  linear_threshold_tag, omp_parallel_tag, sequential_tag)

__version__ = "0.1.0"


def library_version() -> str:
    return _lib.lib.rip_version().decode()


def theta_prime(x: int, epsilon_prime: float, l: float, k: int, n: int) -> int:
    """include/ripples/imm.h:77-85 (ssize_t truncation)."""
    return int(_lib.lib.rip_theta_prime(x, epsilon_prime, l, k, n))


def inv_theta_prime(rr_size: int, epsilon_prime: float, l: float, k: int, n: int) -> int:
    """include/ripples/imm.h:96-105."""
    return int(_lib.lib.rip_inv_theta_prime(rr_size, epsilon_prime, l, k, n))


def theta(epsilon: float, l: float, k: int, lower_bound: float, n: int) -> int:
    """include/ripples/imm.h:114-128 (size_t truncation)."""
    return int(_lib.lib.rip_theta(epsilon, l, k, lower_bound, n))


def log_binomial(n: int, k: int) -> float:
    """include/ripples/utility.h:84-87."""
    return float(_lib.lib.rip_log_binomial(n, k))
