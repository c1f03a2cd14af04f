'''A touching pair of identical spheres (same contract as
theory/Dimer.py): the spheres sit at +-(a_p / magnification) pixels from
the cluster centre along the axis (cos theta cos phi, cos theta sin phi,
sin theta) (theory/Dimer.py:76-90).'''
from dataclasses import dataclass

import numpy as np

from .Cluster import Cluster
from .Sphere import Sphere


@dataclass
class Dimer(Cluster):
    a_p: float = 0.75
    n_p: float = 1.45
    k_p: float = 0.
    theta: float = np.pi / 4.
    phi: float = 0.
    magnification: float = 0.048

    def __post_init__(self):
        p = dict(a_p=self.a_p, n_p=self.n_p, k_p=self.k_p)
        self.particles = [Sphere(**p), Sphere(**p)]
        self.update_positions()

    def __setattr__(self, key, value):
        super().__setattr__(key, value)
        if key in ('a_p', 'n_p', 'k_p'):
            for p in getattr(self, 'particles', []):
                setattr(p, key, value)
        if key in ('a_p', 'theta', 'phi', 'magnification'):
            self.update_positions()

    @property
    def properties(self):
        return {'x_p': self.x_p, 'y_p': self.y_p, 'z_p': self.z_p,
                'a_p': self.a_p, 'n_p': self.n_p, 'k_p': self.k_p,
                'theta': self.theta, 'phi': self.phi}

    @properties.setter
    def properties(self, properties):
        for name, value in properties.items():
            if hasattr(self, name):
                setattr(self, name, value)

    def update_positions(self):
        if len(getattr(self, 'particles', [])) != 2:
            return
        axis = np.array([np.cos(self.theta) * np.cos(self.phi),
                         np.cos(self.theta) * np.sin(self.phi),
                         np.sin(self.theta)])
        offset = (self.a_p / self.magnification) * axis
        self.particles[0].r_p = offset
        self.particles[1].r_p = -offset
