"""openqarp_b200 — a B200-native statevector engine behind the QarpEngine simulator seam.

The hot path (gate application, Pauli-sum expectation, terminal sampling, adjoint
gradients) runs as hand-written sm_100a CUDA kernels in ``libqsv.so``, reached through a
C-ABI (include/qsv.h) with ctypes.  Importing the package loads the library and fails
loudly when it is missing: there is no CPU fallback.
"""
from .errors import CapabilityError, CudaError
from .ir import Command, GateType, Param, custom, gate, pack
from .noise import (NoiseModel, make_amplitude_damping, make_bit_flip, make_depolarizing,
                    make_pauli)
from .observable import PauliMasks, from_strings, to_masks
from .program import Program
from .simulator import B200Simulator, Register, SamplingResult, uniforms

__all__ = [
    "B200Simulator", "Register", "SamplingResult", "uniforms",
    "Command", "GateType", "Param", "custom", "gate", "pack",
    "PauliMasks", "from_strings", "to_masks", "Program",
    "CapabilityError", "CudaError",
    "NoiseModel", "make_depolarizing", "make_pauli", "make_bit_flip", "make_amplitude_damping",
]
