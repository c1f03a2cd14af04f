'''A cluster of particles scattering together (same contract as
theory/Cluster.py): the cluster's position is the origin (r_0) of each
member; the model superposes the members' fields in one kernel item.'''
from dataclasses import dataclass, field

from .Particle import Particle


@dataclass
class Cluster(Particle):
    particles: list = field(repr=False, default_factory=list)

    def __post_init__(self):
        self.update()

    def __setattr__(self, key, value):
        super().__setattr__(key, value)
        if key in ('x_p', 'y_p', 'z_p', 'particles'):
            self.update()

    def __len__(self):
        return len(self.particles)

    def __iter__(self):
        return iter(self.particles)

    def __getitem__(self, index):
        return self.particles[index]

    @property
    def properties(self):
        return {'x_p': self.x_p, 'y_p': self.y_p, 'z_p': self.z_p}

    @properties.setter
    def properties(self, properties):
        Particle.properties.fset(self, properties)

    def update(self):
        '''Propagate the cluster's position to each member's origin.'''
        try:
            for particle in self.particles:
                particle.r_0 = self.r_p
        except AttributeError:
            pass
