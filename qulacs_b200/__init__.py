"""qulacs_b200: the Qulacs state-update path on NVIDIA B200 (sm_100a).

Host API mirroring qulacs' QuantumState / gate / QuantumCircuit / Observable over the C ABI in
``include/qulacs_b200.h``; all computation runs in hand-written CUDA kernels in
``libqulacs_b200.so``.  Importing the package does not load the library; the first object created
does, and raises if it has not been built.
"""
from . import gate
from .circuit import QuantumCircuit
from .noise import NoiseSimulator
from .observable import Observable, PauliOperator
from .state import DensityMatrix, QuantumState, QuantumStateC64, inner_product, set_default_stream

__all__ = [
    "gate", "QuantumCircuit", "Observable", "PauliOperator", "QuantumState", "QuantumStateC64",
    "DensityMatrix", "inner_product", "set_default_stream", "NoiseSimulator",
]
