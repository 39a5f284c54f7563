"""Backend registry (src/backends.jl:24-219): EinsumBackend types and the
global selection set_einsum_backend / get_einsum_backend.

``B200Backend`` is this package's backend and the default here.  The
reference's ``DefaultBackend`` (BLAS/CUBLAS) and ``CuTensorBackend`` exist as
types for API compatibility; they are not implemented by this package, so
contracting with one of them selected raises instead of falling back.
Like the reference, the global selection is not thread-safe
(src/backends.jl:115-117).
"""
from __future__ import annotations


class EinsumBackend:
    """``abstract type EinsumBackend`` (src/backends.jl:24)."""


class DefaultBackend(EinsumBackend):
    """The reference's BLAS/CUBLAS backend (src/backends.jl:53); not provided here."""

    def __repr__(self):
        return "DefaultBackend()"


class CuTensorBackend(EinsumBackend):
    """The reference's cuTENSOR backend (src/backends.jl:105); not provided here."""

    def __repr__(self):
        return "CuTensorBackend()"


class B200Backend(EinsumBackend):
    """The sm_100a backend of this package.

    prec (FP32 only): 0 = AUTO = 3 = BF16X6 (tensor-core products of a 3-term
    bf16 split, FP32-faithful), 1 = FP32 (CUDA-core FP32 everywhere, the
    plain GPU path), 2 = BF16X3 (2-term split: twice as fast, about 16-bit
    products).  Other element types ignore it.
    """

    def __init__(self, prec: int = 0):
        self.prec = int(prec)

    def __repr__(self):
        return f"B200Backend(prec={self.prec})"

    def __eq__(self, other):
        return isinstance(other, B200Backend) and other.prec == self.prec


_BACKEND = [B200Backend()]


def set_einsum_backend(backend: EinsumBackend) -> EinsumBackend:
    """``set_einsum_backend!`` (src/backends.jl:164-167)."""
    if not isinstance(backend, EinsumBackend):
        raise TypeError("expected an EinsumBackend")
    _BACKEND[0] = backend
    return backend


def get_einsum_backend() -> EinsumBackend:
    """``get_einsum_backend`` (src/backends.jl:219)."""
    return _BACKEND[0]
