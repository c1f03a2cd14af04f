from .Particle import Particle
from .Sphere import Sphere
from .Instrument import Instrument
from .LorenzMie import LorenzMie

LMHologram = LorenzMie

__all__ = ['Particle', 'Sphere', 'Instrument', 'LorenzMie', 'LMHologram']
