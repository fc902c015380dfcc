"""B200 (sm_100a) implementation of FlexRT's per-timestep radiative-transfer path.

The RT step (HEALPix ray casting with split/merge, the per-frequency optical-depth walk with
Gamma deposition, the C2Ray cell update, the thermal update and dt) runs as CUDA kernels behind the
C ABI in include/flexrt.h (lib/libflexrt_b200.so). `rt.RTContext` mirrors the reference's
rt_funcs/ray_tracing call surface on top of that ABI; `workloads` builds the seeded synthetic boxes.
"""
from . import workloads  # noqa: F401

__all__ = ["workloads", "rt", "build"]
