"""bridct_b200: B200-native (sm_100a) orthonormal 2D DCT-II / DCT-III / round trip.

Drop-in surfaces of the reference's hot path:
  * C plan API (include/bridct.h) in libbridct_b200.so, plus B200 extensions
    (include/bridct_b200.h);
  * ``bridct_b200.bridct_numpy.Plan`` - the reference NumPy contract;
  * ``bridct_b200.torch_api`` - CUDA tensors, autograd, precision forms.
"""
from . import _lib

__version__ = _lib.VERSION
core_version = _lib.VERSION


def supported(height: int, width: int) -> bool:
    return bool(_lib.lib().bridct_supported(int(height), int(width)))
