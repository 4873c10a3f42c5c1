"""parallel-RA's semi-naive fixed point on one B200.

The engine is native: CUDA kernels for sm_100a plus a C ABI
(include/ra_engine.h) in ``libra_b200.so``, and the reference's C++ classes
(relation, RAM, parallel_join, parallel_copy, parallel_copy_filter, LIE) in
``libparallel_ra.so``.  This Python package is a ctypes binding of the C ABI
(``engine``), the TC / SG program definitions (``programs``), seeded input
generators (``datagen``), batched execution of many instances per launch
(``batch``) and transitive closure partitioned over ranks (``partition``).
"""
from . import batch, datagen, engine, partition, programs  # noqa: F401
from .engine import Program, RAError  # noqa: F401

__all__ = ["Program", "RAError", "batch", "datagen", "engine", "partition", "programs"]
