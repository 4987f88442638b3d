"""sfparticles_b200 -- a B200-native implementation of the sfparticles
per-particle step, with the reference's Python API (sfparticles/__init__.py:1-5).

    from sfparticles_b200 import Particles, SpinParticles, Simulation, Fields, RadiationReactionType
    from sfparticles_b200.fields import gaussian_laser_pulse

All computation runs in libsfp.so (hand-written CUDA for sm_100a, loaded
through a C-ABI); there is no CPU code path.  ``SFPARTICLES_USE_GPU`` is
accepted for compatibility and must not be "0".
"""
from os import getenv as _getenv

if _getenv("SFPARTICLES_USE_GPU", "1") == "0":
    raise ImportError("sfparticles_b200 is the GPU implementation; SFPARTICLES_USE_GPU=0 selects the reference's "
                      "CPU path, which this package does not contain")

from .fields import Fields  # noqa: E402
from .particles import Particles, RadiationReactionType, SpinParticles  # noqa: E402
from .simulation import Simulation  # noqa: E402
from .ensemble import Ensemble  # noqa: E402

_use_gpu = True
__all__ = ["Particles", "SpinParticles", "Simulation", "Ensemble", "Fields", "RadiationReactionType"]
__version__ = "0.1.0"
