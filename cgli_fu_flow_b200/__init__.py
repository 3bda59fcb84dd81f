"""B200 implementation of the CGLI_Fu_Flow per-step hot path.

The compute path is libcgli_fu_flow.so (hand-written CUDA for sm_100a behind
the C ABI of include/cgli_fu_flow.h); this package holds its build recipe,
the Python mirror of the reference's routine interface and the channel
workload definitions.
"""
from .channel import Channel, WORKLOADS  # noqa: F401

__all__ = ["Channel", "WORKLOADS"]
