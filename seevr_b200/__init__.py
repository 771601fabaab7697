"""seevr_b200 — sm_100a rigid-body physics step with the dispatch API and
buffer layout of seeVR's physics.comp / physics.zig.

The compute path is libseevr_cuda.so (C ABI in include/seevr.h); importing
this package fails if that library is not built.
"""
from ._lib import (SeevrError, Profile, STAGE_NAMES, SOLVER_SEQUENTIAL, SOLVER_WAVEFRONT,
                   SOLVER_COLORED, BROADPHASE_N2, BROADPHASE_LBVH, FLAG_NO_SYNC,
                   FLAG_CUDA_GRAPH, FLAG_SKIP_RENDER_VERTS, LIB_PATH, NARROWPHASE_MPR,
                   NARROWPHASE_GJK_EPA)
from .data import Caps, Data, DeviceBuffers
from .physics import Physics, make_params

__all__ = [
    "Caps", "Data", "DeviceBuffers", "Physics", "make_params", "SeevrError", "Profile",
    "STAGE_NAMES", "SOLVER_SEQUENTIAL", "SOLVER_WAVEFRONT", "SOLVER_COLORED", "BROADPHASE_N2",
    "BROADPHASE_LBVH", "FLAG_NO_SYNC", "FLAG_CUDA_GRAPH", "FLAG_SKIP_RENDER_VERTS", "LIB_PATH",
    "NARROWPHASE_MPR", "NARROWPHASE_GJK_EPA",
]
