"""libsci_b200: a B200 (sm_100a) CUDA backend for libsci's fused-expression, reduction,
product and LU/solve paths, behind a C ABI (include/sci_cuda.h).

``libsci_b200.chunk`` restates libsci's chunk bytecode and recorder; ``libsci_b200.device``
is the host layer over libsci_cuda.so (imported lazily, so the recorder works without a GPU
build). Importing ``libsci_b200.device`` without the built library raises.
"""
from . import chunk  # noqa: F401

__all__ = ["chunk"]
