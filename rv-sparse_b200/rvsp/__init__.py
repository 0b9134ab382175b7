"""rv-sparse-b200: B200-native CSR SpGEMM behind the rv-sparse C API.

The product is the C-ABI library lib/librvsparse_cuda.so (hand-written
sm_100a kernels + a C11 host layer).  This package is its Python mirror for
tests and benchmarks: ctypes bindings (`_lib`), a host CSR container
(`csr`), the API wrappers (`api`) and seeded workload generators (`gen`).
"""
from . import _lib as lib
from ._lib import RvspError, check, load
from .api import Batch, Descriptor, DeviceCSR, read_mtx, spgemm_csr, spgemm_typed
from .csr import CSR, algorithmic_bytes, intermediate_products

__all__ = ["lib", "RvspError", "check", "load", "Batch", "Descriptor", "DeviceCSR",
           "read_mtx", "spgemm_csr", "spgemm_typed", "CSR", "algorithmic_bytes", "intermediate_products"]
