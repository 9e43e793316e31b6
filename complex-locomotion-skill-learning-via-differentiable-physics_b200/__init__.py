"""B200-native differentiable soft-robot simulation step.

Fused sm_100a CUDA kernels (mass-spring solver + MLP controller, forward and
hand-written adjoint, checkpointed recompute; MLS-MPM) behind the C ABI in
``include/cls_b200.h``.  Host modules: ``batch`` (the batch front-end),
``trainer`` (the reference trainer's interface), ``dropin`` (duck-typed
stand-ins for the reference's TaichiEnv / SolverMassSpring / Model objects),
``clients`` (headless interactive and gym clients), ``serving`` (request
loop), ``sharding`` (shared controllers across GPUs), ``mpm``.
"""
from . import _capi
from .batch import MassSpringBatch, Robot, default_params

__all__ = ["MassSpringBatch", "Robot", "default_params", "_capi"]
