"""strata_b200 — B200 relational fixpoint engine for Strata/K's semi-naive hot path.

``gpu``      the reference GPU crate's API (transitive_closure_bool, …) on CUDA.
``ops``      the interpreter's rule evaluation composed from the device
             operator surface (select / join / intersect / semijoin /
             project / sort / reduce / merge-diff / aggregate).
``gen``      seeded synthetic inputs of the benchmark shapes.
``textio``   the TSV input contract and the canonical text renderer.
"""
from . import _lib  # noqa: F401
from .gpu import (  # noqa: F401
    POS_INF, BatchResult, BoolRelation, Cuda, DeviceRelation, Engine, GpuError, InvalidArgument,
    NegativeWeightCycle, NotBuilt, OutOfMemory, Timeout, TropOverflow, TropRelation, Unsupported,
    WeightRange, binary_plan_intermediate, count_4cliques, count_triangle_pattern, count_triangles,
    default_engine, intern_terms, mssp_trop, shortest_paths_trop, transitive_closure_bool,
)

__version__ = "0.1.0"
