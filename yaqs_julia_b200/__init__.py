"""B200 (sm_100a) tensor-jump-method trajectory engine with the Yaqs.jl API.

The compute path is libyaqs_b200.so (CUDA, built in-tree); this package is
its host-side mirror of the reference's interface (api.py) and the ctypes
binding of the C-ABI in include/yaqs_tjm.h (_abi.py, _lib.py).
"""
from .api import (MPO, MPS, NoiseModel, Observable, TimeEvolutionConfig, init_general_hamiltonian,  # noqa: F401
                  init_ising, run)
