"""fwi3d_b200: B200-native (sm_100a) time-stepping wave propagation and adjoint
gradients with the operator interface of nmbader/fwi3d.

The compute path is libfwi3d_b200.so (CUDA kernels + C ABI, include/fwi3d_gpu.h);
this package is its host-side mirror of the reference's nl_we_op_* operators.
"""
from .param import Param  # noqa: F401

__all__ = ["Param", "ops", "synth"]
