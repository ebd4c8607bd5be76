"""B200 implementation of Sedona's implicit Monte Carlo transport step.

The compute path is the CUDA library pubsed_b200/libsedona_gpu.so behind the C
ABI in include/sedona_gpu.h; this package holds the host-side mirror of the
reference `transport` interface (pubsed_b200.transport), the Lua parameter
interface (pubsed_b200.params) and the synthetic workloads used by the tests
and the benchmark (pubsed_b200.workloads).
"""
__all__ = ["abi", "grids", "params", "atomic", "workloads"]
