"""B200-native differentiable soft-robot simulation step.

Fused sm_100a CUDA kernels (mass-spring solver + MLP controller, forward and
hand-written adjoint, checkpointed recompute) behind the C ABI in
``include/cls_b200.h``, with host classes that mirror the reference's
solver / env / model interface.
"""
from . import _capi
from .batch import MassSpringBatch, Robot, default_params

__all__ = ["MassSpringBatch", "Robot", "default_params", "_capi"]
