"""Reference-shaped host API of the IMM hot path.

Mirrors the C++ surface of pnnl/ripples that this package replaces, with the
same names and argument meaning:

* :class:`IMMConfiguration` -- ``ToolConfiguration<IMMConfiguration>``
  (include/ripples/configuration.h:56-185, imm_configuration.h:63-176): the
  ``-k``, ``-e``, ``-d``, ``-p`` options and the streaming knobs.
* :class:`IMMExecutionRecord` -- include/ripples/imm_execution_record.h:55-92,
  serialised with the JSON keys of tools/imm.cc:104-134.
* :class:`B200RRRGenerator` -- the generator object handed to ``IMM`` in place
  of ``StreamingRRRGenerator`` (include/ripples/streaming_rrr_generator.h:833).
* :func:`GenerateRRRSets`, :func:`FindMostInfluentialSet`, :func:`IMM` --
  include/ripples/generate_rrr_sets.h:186-224,
  include/ripples/find_most_influential.h:85-196, include/ripples/imm.h:671-860.

Everything computes on the GPU through the native library; errors surface as
:class:`ripples_b200._lib.RipError` (the reference throws ``std::logic_error``
/ ``std::domain_error`` or exits).
"""
from __future__ import annotations

import json
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple, Union

import numpy as np

from . import _lib
from .graph import Context, DeviceGraph, HostGraph, Pool


class independent_cascade_tag:  # noqa: N801 - reference spelling
    name = "IC"


class linear_threshold_tag:  # noqa: N801
    name = "LT"


class sequential_tag:  # noqa: N801
    pass


class omp_parallel_tag:  # noqa: N801
    pass


@dataclass
class IMMConfiguration:
    k: int = 10
    epsilon: float = 0.5
    diffusionModel: str = "IC"  # noqa: N815 - reference field name
    parallel: bool = True
    IFileName: str = ""  # noqa: N815
    OutputFile: str = "output.json"  # noqa: N815
    num_rr_sets: int = 0
    seed_select_max_workers: int = 0
    seed_select_max_gpu_workers: int = 0
    gpu_batch_size: int = 64  # fused colour width (64/128/256)
    streaming_gpu_workers: int = 1
    streaming_workers: int = 1
    streaming_cpu_teams: int = 0
    pause_threshold: float = 1.0
    # B200 additions
    tiebreak: int = _lib.TIE_REF_HEAP
    sampler: int = _lib.SAMPLER_AUTO
    seed: int = 0


@dataclass
class IMMExecutionRecord:
    NumThreads: int = 1
    Total: float = 0.0
    ThetaPrimeDeltas: List[int] = field(default_factory=list)
    ThetaEstimationTotal: float = 0.0
    ThetaEstimationGenerateRRR: List[float] = field(default_factory=list)
    ThetaEstimationMostInfluential: List[float] = field(default_factory=list)
    Theta: int = 0
    Counting: List[float] = field(default_factory=list)
    Pivoting: List[float] = field(default_factory=list)
    Microbenchmarking: float = 0.0
    CPUBatchSize: int = 0
    GPUBatchSize: int = 64
    RRRSetSize: int = 0
    GenerateRRRSets: float = 0.0
    FindMostInfluentialSet: float = 0.0
    # B200 additions
    TotalSets: int = 0
    PoolElements: int = 0
    F: float = 0.0

    @classmethod
    def from_native(cls, r: _lib.ImmRecord, gpu_batch: int) -> "IMMExecutionRecord":
        nr = min(r.num_rounds, _lib.MAX_ROUNDS)
        return cls(
            Total=r.total_ms,
            ThetaPrimeDeltas=[int(r.theta_prime_deltas[i]) for i in range(nr)],
            ThetaEstimationTotal=r.theta_estimation_ms,
            ThetaEstimationGenerateRRR=[r.round_generate_ms[i] for i in range(nr)],
            ThetaEstimationMostInfluential=[r.round_select_ms[i] for i in range(nr)],
            Theta=int(r.theta),
            GPUBatchSize=gpu_batch,
            RRRSetSize=int(r.rrr_set_bytes),
            GenerateRRRSets=r.generate_ms,
            FindMostInfluentialSet=r.select_ms,
            TotalSets=int(r.total_sets),
            PoolElements=int(r.pool_elements),
            F=r.f,
        )

    def experiment(self, CFG: IMMConfiguration, seeds: Sequence[int]) -> dict:
        """One entry of the imm tool's JSON log (tools/imm.cc:101-136)."""
        return {
            "Algorithm": "IMM",
            "Input": CFG.IFileName,
            "Output": CFG.OutputFile,
            "DiffusionModel": CFG.diffusionModel,
            "Epsilon": CFG.epsilon,
            "K": CFG.k,
            "L": 1,
            "NumThreads": self.NumThreads,
            "NumWalkWorkers": CFG.streaming_workers,
            "NumCPUTeams": CFG.streaming_cpu_teams,
            "NumGPUWalkWorkers": CFG.streaming_gpu_workers,
            "PauseThreshold": CFG.pause_threshold,
            "Total": self.Total,
            "ThetaPrimeDeltas": self.ThetaPrimeDeltas,
            "ThetaEstimation": self.ThetaEstimationTotal,
            "ThetaEstimationGenerateRRR": self.ThetaEstimationGenerateRRR,
            "ThetaEstimationMostInfluential": self.ThetaEstimationMostInfluential,
            "Theta": self.Theta,
            "Counting": self.Counting,
            "Pivoting": self.Pivoting,
            "Microbenchmarking": self.Microbenchmarking,
            "CPUBatchSize": self.CPUBatchSize,
            "GPUBatchSize": self.GPUBatchSize,
            "RRRSetSizeBytes": self.RRRSetSize,
            "GenerateRRRSets": self.GenerateRRRSets,
            "FindMostInfluentialSet": self.FindMostInfluentialSet,
            "Seeds": [int(s) for s in seeds],
        }


class B200RRRGenerator:
    """Generator object for :func:`IMM` / :func:`GenerateRRRSets`: a graph
    resident in HBM plus a device RRR pool.  Set ``i`` of the pool is a pure
    function of (graph, seed, i)."""

    def __init__(self, G: HostGraph, model: str, seed: int = 0, device: int = 0,
                 ctx: Optional[Context] = None, colors: int = 64,
                 sampler: int = _lib.SAMPLER_AUTO):
        self.ctx = ctx or Context(device)
        self.graph = DeviceGraph(self.ctx, G, model)
        self.pool = Pool(self.graph)
        self.pool.configure(colors=colors)
        self.seed, self.model, self.sampler, self.colors = seed, model, sampler, colors

    def isGpuEnabled(self) -> bool:  # noqa: N802 - reference name
        return True

    def generate(self, count: int, record: Optional[IMMExecutionRecord] = None) -> None:
        self.pool.sample(count, self.seed, self.sampler)

    def sets(self, first: int = 0, count: Optional[int] = None) -> List[np.ndarray]:
        off, vtx = self.pool.export(first, count)
        return [vtx[off[i]:off[i + 1]] for i in range(len(off) - 1)]


def _as_csr(RR: Sequence[Sequence[int]]) -> Tuple[np.ndarray, np.ndarray]:
    lens = np.fromiter((len(s) for s in RR), dtype=np.uint64, count=len(RR))
    off = np.zeros(len(RR) + 1, dtype=np.uint64)
    np.cumsum(lens, out=off[1:])
    vtx = np.concatenate([np.asarray(s, dtype=np.uint32) for s in RR]) if len(RR) else \
        np.zeros(0, dtype=np.uint32)
    return off, vtx


def GenerateRRRSets(G: HostGraph, generator: B200RRRGenerator, RR: Optional[list],
                    count: int, record: Optional[IMMExecutionRecord] = None,
                    model_tag=None, ex_tag=None) -> None:  # noqa: N802
    """Appends ``count`` RRR sets (sorted ascending) to the generator's pool
    and, when ``RR`` is a list, to ``RR`` as numpy arrays -- the reference fills
    caller-provided empty sets (include/ripples/generate_rrr_sets.h:186-224)."""
    first = generator.pool.num_sets
    generator.generate(count, record)
    if RR is not None:
        RR.extend(generator.sets(first, count))


def FindMostInfluentialSet(G, CFG: IMMConfiguration, RR: Union[Pool, B200RRRGenerator, Sequence],
                           record: Optional[IMMExecutionRecord] = None,
                           enableGPU: bool = True, ex_tag=None,
                           num_sets: Optional[int] = None,
                           ctx: Optional[Context] = None) -> Tuple[float, List[int]]:  # noqa: N802,N803
    """Greedy max coverage over RRR sets; returns ``(f, seeds)`` like
    include/ripples/find_most_influential.h:176-196.  ``RR`` is a device pool,
    a generator, or a host list of sets (uploaded to a temporary pool)."""
    if isinstance(RR, B200RRRGenerator):
        RR = RR.pool
    if isinstance(RR, Pool):
        f, seeds, _ = RR.select(CFG.k, num_sets, CFG.tiebreak)
        return f, [int(s) for s in seeds]
    assert isinstance(G, HostGraph)
    own = ctx is None
    ctx = ctx or Context()
    g = HostGraph(G.n, G.index, G.src, G.weights if G.weights is not None else
                  np.zeros(G.m, dtype=np.float32))
    dg = DeviceGraph(ctx, g, CFG.diffusionModel)
    pool = Pool(dg)
    try:
        off, vtx = _as_csr(RR)
        pool.import_sets(off, vtx)
        f, seeds, _ = pool.select(CFG.k, num_sets, CFG.tiebreak)
        return f, [int(s) for s in seeds]
    finally:
        pool.close()
        dg.close()
        if own:
            ctx.close()


def IMM(G: HostGraph, CFG: IMMConfiguration, l: float, generator: B200RRRGenerator,
        record: Optional[IMMExecutionRecord] = None, model_tag=None,
        ex_tag=None) -> List[int]:  # noqa: N802
    """IMM on one B200 (include/ripples/imm.h:768-860): martingale theta
    estimation, final sampling, final selection over sets [0, theta).
    Returns the seed vertices (internal ids; the binary format's reverse map
    is the identity for graphs built here)."""
    seeds, rec = generator.pool.imm(CFG.k, CFG.epsilon, l, generator.seed, CFG.tiebreak,
                                    generator.sampler)
    if record is not None:
        r = IMMExecutionRecord.from_native(rec, generator.colors)
        record.__dict__.update(r.__dict__)
    return [int(s) for s in seeds]


def write_log(path: str, CFG: IMMConfiguration, record: IMMExecutionRecord,
              seeds: Sequence[int]) -> None:
    with open(path, "w") as fh:
        json.dump([record.experiment(CFG, seeds)], fh, indent=2)
