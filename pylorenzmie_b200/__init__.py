'''pylorenzmie_b200: the Lorenz-Mie hologram model and its fitting loop on
NVIDIA B200 (sm_100a), behind pylorenzmie's LorenzMie / Optimizer API.

The compute is a C-ABI CUDA library (include/lmb200.h,
pylorenzmie_b200/csrc); this package is its host-side mirror of the
reference interface.  Importing the package does not touch the GPU.
'''
__version__ = '0.1.0'

from .lib import meshgrid, LMObject  # noqa: F401
from .theory import (Particle, Sphere, LayeredSphere, Cluster,  # noqa: F401
                     Dimer, Instrument, LorenzMie, Aberrated,
                     AberratedLorenzMie)
from .analysis import (Hologram, Mask, Optimizer, DEEstimator,  # noqa: F401
                       RadialEstimator, Feature, Frame)
