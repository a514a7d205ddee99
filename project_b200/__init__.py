"""B200-native ERK4(3) interaction-picture UPPE/GNLSE propagator.

Drop-in for the propagate path of the reference's 1D gas solver
(``ERK43IP_UPPE``) and 3+1D envelope solver (``ERK43IP_UPPE_3D_Optimized``):
Python host code computes the FP64 setup tables, hand-written sm_100a CUDA
kernels in ``libuppe_b200.so`` do every per-step operation.  No CPU fallback.
"""
from .media import Argon, OpticalMedium, adk_rate  # noqa: F401


def __getattr__(name):
    if name == 'ERK43IP_UPPE_3D_Optimized':
        from .solver3d import ERK43IP_UPPE_3D_Optimized
        return ERK43IP_UPPE_3D_Optimized
    raise AttributeError(name)
