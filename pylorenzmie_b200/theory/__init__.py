from .Particle import Particle
from .Sphere import Sphere
from .LayeredSphere import LayeredSphere
from .Cluster import Cluster
from .Dimer import Dimer
from .Instrument import Instrument
from .LorenzMie import LorenzMie
from .Aberrated import Aberrated, AberratedLorenzMie

LMHologram = LorenzMie

__all__ = ['Particle', 'Sphere', 'LayeredSphere', 'Cluster', 'Dimer',
           'Instrument', 'LorenzMie', 'Aberrated', 'AberratedLorenzMie',
           'LMHologram']
