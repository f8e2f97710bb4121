"""parbutterfly_b200 — B200-native (sm_100a) butterfly counting and peeling for bipartite graphs.

A drop-in for ParButterfly's wedge-aggregation hot path (apps/hyper/BipartiteButterflies.C and
the butterfly_*.h algorithms): the same option surface (count / rank / peel / per types), the
same input format, bit-exact results, computed by hand-written CUDA kernels behind the C ABI in
include/parbutterfly_b200.h.
"""
from .graph import BipartiteGraph, workload  # noqa: F401
