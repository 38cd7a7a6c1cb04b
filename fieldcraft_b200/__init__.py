"""fieldcraft_b200: the numeric phase of FieldCraft's supernodal sparse Cholesky (the direct solve
behind its implicit FEM analyses, K u = f) rebuilt for NVIDIA B200, behind the reference's own
factorise/solve API. See include/fieldcraft_chol.h for the C ABI."""
from .cholesky import (FP32_IR, FP64, LDLT, Cancelled, Csr, DeviceError, Factor, FactorError, Inertia, Internal,
                       Kind, LdltFactor, NotPositiveDefinite, OutOfMemory, Singular, Symbolic, Symmetric, Timeout,
                       TooLarge, UpperColumns)

__all__ = ["Csr", "UpperColumns", "Symbolic", "Factor", "FactorError", "NotPositiveDefinite", "Singular",
           "TooLarge", "OutOfMemory", "Internal", "Cancelled", "Timeout", "DeviceError", "FP64", "FP32_IR", "LDLT",
           "LdltFactor", "Inertia", "Symmetric", "Kind"]
