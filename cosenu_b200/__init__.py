"""B200-native (sm_100a) RK4 time-stepping path for COSEnu.

The CUDA library (``libcosenu_b200.so``, C ABI in ``include/cosenu_b200.h``)
holds the state on the GPU and advances it with fused RK4 stage kernels;
``NuOsc`` is its Python face, shaped like the reference's NuOsc class.
"""
from .nuosc import NuOsc, make_params, COMPONENTS  # noqa: F401

__all__ = ["NuOsc", "make_params", "COMPONENTS"]
