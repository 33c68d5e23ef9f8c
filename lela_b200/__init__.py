"""lela_b200 -- B200 (sm_100a) implementation of LELA's exact linear-algebra
hot path: dense gemm/trsm over Z/p (Modular<uint32>) and GF(2), dense
echelon forms, and the Faugere-Lachartre echelonization built on them.

The compute lives in hand-written CUDA (``lela_b200/csrc``) behind the C ABI
of ``include/lela_cuda.h``, built into ``lela_b200/liblela_cuda.so``.  This
package is the Python host mirror of LELA's interface for that path: the
same operation names, argument meaning and exceptions (see ``api``).  There
is no CPU fallback: if the CUDA library is missing or no B200 is visible,
every operation raises.
"""
from .api import (  # noqa: F401
    CudaModule,
    LELAError,
    DiagonalEntryNotInvertible,
    WrongMatrixForm,
    PreconditionFailed,
    CudaError,
    load_library,
    library_path,
)
