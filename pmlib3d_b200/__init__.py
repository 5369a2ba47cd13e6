"""B200 implementation of pmlib3d's particle-mesh vortex step.

The product is the CUDA library ``libpmgpu.so`` (C ABI in ``include/pmlib_gpu.h``);
``pmlib3d_b200.pmlib`` mirrors the reference's module procedures on top of it.
"""
from . import pmlib  # noqa: F401
