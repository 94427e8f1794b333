"""cugip_b200: B200-native grid graph-cut (exact push-relabel max-flow/min-cut).

The compute path is libcgc.so (hand-written sm_100a CUDA behind the C ABI of
include/cgc.h); this package is its host-side mirror of cugip's Graph API.
"""
from ._lib import CgcError, load  # noqa: F401
from .graph_cut import SINK, SOURCE, Batch, GenericGraph, Graph, GridGraph, Policy  # noqa: F401

__all__ = ["CgcError", "load", "Graph", "GridGraph", "Batch", "Policy", "SINK", "SOURCE"]
