"""zinq_b200: a B200-native split-operator wavepacket propagator.

Drop-in for the grid quantum-dynamics path of Zinq (src/quantum_dynamics.zig):
the same options and observables, computed by hand-written sm_100a CUDA
kernels behind the C-ABI declared in include/zinq_qd.h (libzinq_qd.so).
"""
from ._abi import ZqdError  # noqa: F401

__all__ = ["ZqdError", "quantum_dynamics", "build"]
