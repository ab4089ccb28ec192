"""B200-native multispin-coded Ising spin-glass Metropolis engine.

The compute path is libsa_b200.so (hand-written CUDA for sm_100a behind the C
ABI in include/sa_b200.h); this package is its Python host side: the gpu_sys
mirror (GpuSystem), the annealing / parallel-tempering drivers, the batched
engine and the serving loop.
"""
from ._lib import SAError, load  # noqa: F401

__all__ = ["SAError", "load"]
