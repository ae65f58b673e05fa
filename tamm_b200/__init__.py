"""tamm_b200 — B200-native block-sparse tensor contractions with TAMM's API.

The compute path is libtamm_b200.so (hand-written sm_100a kernels behind the C ABI
in include/tamm_b200.h); this package is a thin Python front-end over it.
"""
from ._capi import TambError, lib, last_error  # noqa: F401
from .tamm import (ExecutionContext, ExecutionHW, IndexSpace, LabeledTensor, Map, Precision,  # noqa: F401
                   Scheduler, Tape, Tensor, TiledIndexLabel, TiledIndexSpace, apply_ewise_ip)

__all__ = ["ExecutionContext", "ExecutionHW", "IndexSpace", "LabeledTensor", "Map", "Precision", "apply_ewise_ip",
           "Scheduler", "Tape", "Tensor", "TiledIndexLabel", "TiledIndexSpace", "TambError", "lib",
           "last_error"]
