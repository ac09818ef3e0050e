"""flexpart_gpu — host side of the B200 backend for the flexpart-gpu
per-particle timestep.  Compute runs in libfpg.so (CUDA, sm_100a) through the
C ABI declared in include/fpg.h; this package holds the ctypes binding, the
reference-shaped host objects and the synthetic inputs of the benchmark
configurations."""
from .records import (  # noqa: F401
    FLAG_ACTIVE,
    MAX_SPECIES,
    PARTICLE_DTYPE,
    SURFACE_DTYPE,
    PblOptions,
    StepParams,
)
