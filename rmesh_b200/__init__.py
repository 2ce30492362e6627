"""B200-native implementation of rmeshvk's differentiable tiled tet-mesh volume
rendering path: per-tet projection and culling, tile binning, onesweep radix
sorts, tiled front-to-back compositing, loss, recompute-based adjoint and fused
Adam, as hand-written sm_100a CUDA behind the C ABI in include/rmesh_b200.h.

``RMeshRenderer`` mirrors the reference's PyO3 class; ``RMeshForward`` and
``RMeshModule`` mirror its torch autograd wrapper.
"""
from .renderer import RMeshError, RMeshRenderer
from .staging import TargetStager

__all__ = ["RMeshRenderer", "RMeshError", "RMeshForward", "RMeshModule", "TargetStager"]


def __getattr__(name):
    # torch is only imported when the autograd wrapper is requested
    if name in ("RMeshForward", "RMeshModule"):
        from . import autograd

        return getattr(autograd, name)
    raise AttributeError(name)
