from .Particle import Particle
from .Sphere import Sphere
from .LayeredSphere import LayeredSphere
from .Instrument import Instrument
from .LorenzMie import LorenzMie

LMHologram = LorenzMie

__all__ = ['Particle', 'Sphere', 'LayeredSphere', 'Instrument', 'LorenzMie',
           'LMHologram']
