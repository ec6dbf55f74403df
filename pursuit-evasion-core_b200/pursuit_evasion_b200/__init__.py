"""B200-native game-value solver for reversible-car pursuit-evasion.

Drop-in for pursuit-evasion-core's relative 5D capture-tube solve
(`reversible.free_dp.solve`) with the per-cell work in hand-written sm_100a
CUDA kernels behind a C ABI (include/pe_b200.h, libpe_b200.so).
"""

__all__ = ["reversible"]
