"""cytnx_b200 -- B200-native (sm_100a) implementation of Cytnx's tensor-network hot path.

Drop-in names of the reference's Python API for that path:
``Type``, ``Device``, ``Symmetry``, ``Bond`` (``BD_KET``/``BD_BRA``/``BD_IN``/``BD_OUT``),
``Tensor``, ``UniTensor``, ``Contract``, ``Network``, ``LinOp``, ``linalg.Lanczos`` and friends.
Compute runs on CUDA devices through ``libcytnx_b200.so`` (hand-written sm_100a kernels
behind the C ABI of include/cytnx_b200.h); there is no CPU compute path.
"""
from . import linalg  # noqa: F401
from ._lib import CytnxError
from .core import (BD_BRA, BD_IN, BD_KET, BD_NONE, BD_OUT, BD_REG, Bond, Device, Symmetry, Tensor, Type,
                   arange, bondType, zeros)
from .batch import BatchedTwoSiteHeff
from .heff import TwoSiteHeff
from .network import LinOp, Network
from .unitensor import Contract, UniTensor, UTenType

Qs = lambda *q: list(q)  # noqa: E731  (cytnx.Qs(...) helper of the reference tests)

__all__ = ["Type", "Device", "Symmetry", "Bond", "BD_KET", "BD_BRA", "BD_IN", "BD_OUT", "BD_REG", "BD_NONE",
           "bondType", "Tensor", "UniTensor", "UTenType", "Contract", "Network", "LinOp", "linalg",
           "TwoSiteHeff", "BatchedTwoSiteHeff", "CytnxError", "arange", "zeros", "Qs"]
