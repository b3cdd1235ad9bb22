"""B200-native MPM substep with slosh's pipeline API.

The device path is ``slosh_b200/lib/libslosh_b200.so`` (hand-written sm_100a
CUDA behind the C ABI of ``include/slosh_b200.h``); this package is the host
side: ctypes binding, the pipeline API mirror and scene generators.
"""
from .pipeline import (  # noqa: F401
    DruckerPrager,
    ElasticCoefficients,
    GpuBoundaryCondition,
    MpmData,
    MpmPipeline,
    ParticleModel,
    RigidBody,
    SimulationParams,
    make_particles,
)
from ._lib import PARTICLE_DTYPE, BODY_DTYPE, SloshError  # noqa: F401
