"""rslab_b200 — B200-native (sm_100a) supernodal LDL^T factor + solve behind
RSLAB's LdltSymbolic / LdltSolver / SolverSettings / MixedLdltSolver API.

The numeric work runs in the in-tree CUDA library librslab_b200.so (C ABI in
include/rslab_b200.h); importing this package fails if it is missing.
"""
from .solver import (  # noqa: F401
    CERT_FACTOR, CompressedLdltFactors, CscMatrix, CudaError, Diagnostics, MemoryEstimate, DimensionMismatch, Inertia, InvalidInput, LdltFactors,
    LdltSolver, LdltSymbolic, MixedInfo, MixedLdltSolver, NumericallyRankDeficient, Ordering, RslabError,
    SolverSettings, ZeroPivotAction, amd_order, device_count,
)
from .ldlt import Ldlt, ldlt  # noqa: F401

__all__ = [
    "CscMatrix", "LdltSymbolic", "LdltSolver", "MixedLdltSolver", "SolverSettings", "ZeroPivotAction",
    "Ordering", "Inertia", "MixedInfo", "LdltFactors", "Diagnostics", "RslabError",
    "NumericallyRankDeficient", "InvalidInput", "DimensionMismatch", "CudaError", "amd_order",
    "device_count", "CERT_FACTOR", "ldlt", "Ldlt", "CompressedLdltFactors", "MemoryEstimate",
]
