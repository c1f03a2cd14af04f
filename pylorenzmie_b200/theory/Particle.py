'''Scattering particle base (same contract as theory/Particle.py).'''
from dataclasses import dataclass, field

import numpy as np

from ..lib import LMObject


@dataclass
class Particle(LMObject):
    '''Position (pixels) and local origin of a particle.

    Implements the sequence protocol so that one particle and a list of
    particles are interchangeable (theory/Particle.py:50-59).
    '''
    x_p: float = 0.
    y_p: float = 0.
    z_p: float = 100.
    x_0: float = field(repr=False, default=0.)
    y_0: float = field(repr=False, default=0.)
    z_0: float = field(repr=False, default=0.)

    def __len__(self):
        return 1

    def __iter__(self):
        return iter([self])

    def __getitem__(self, index):
        if index != 0:
            raise IndexError('Particle index out of range')
        return self

    @property
    def r_p(self):
        return np.asarray([self.x_p, self.y_p, self.z_p])

    @r_p.setter
    def r_p(self, r_p):
        self.x_p, self.y_p, self.z_p = r_p

    @property
    def r_0(self):
        return np.asarray([self.x_0, self.y_0, self.z_0])

    @r_0.setter
    def r_0(self, r_0):
        self.x_0, self.y_0, self.z_0 = r_0

    @LMObject.properties.getter
    def properties(self):
        return {'x_p': self.x_p, 'y_p': self.y_p, 'z_p': self.z_p}
