'''Multilayer (core-shell) sphere.

The reference computes layered coefficients only in dead code
(lib/obsolete/sphere_coefficients.py:65-220, whose list input handling is
broken; it takes ascending radii and one index per layer).  Here the
particle keeps the six fit parameters of a Sphere -- position, outer radius
a_p and the outer layer's index n_p + i k_p -- and describes the inner
layers by their radii as fractions of a_p and their complex indices, so a
fit varies the outer radius with the layer proportions fixed.
'''
from dataclasses import dataclass, field

import numpy as np

from .Sphere import Sphere


@dataclass
class LayeredSphere(Sphere):
    '''Sphere with inner layers.

    fractions    : inner layer radii / a_p, ascending, each in (0, 1)
    core_indices : complex refractive indices of the inner layers, core first
    '''
    fractions: tuple = field(default=(0.5,))
    core_indices: tuple = field(default=(1.5 + 0j,))

    def __post_init__(self):
        self.fractions = tuple(float(f) for f in np.atleast_1d(self.fractions))
        self.core_indices = tuple(complex(c) for c in
                                  np.atleast_1d(self.core_indices))
        if len(self.fractions) != len(self.core_indices):
            raise ValueError('one index per inner layer')
        f = np.asarray(self.fractions)
        if np.any(f <= 0.) or np.any(f >= 1.) or np.any(np.diff(f) <= 0.):
            raise ValueError('fractions must ascend inside (0, 1)')

    @property
    def nlayers(self):
        return len(self.fractions) + 1

    @property
    def radii(self):
        '''Layer radii in um, core first.'''
        return np.array([*(f * self.a_p for f in self.fractions), self.a_p])

    @property
    def indices(self):
        '''Layer indices (complex), core first.'''
        return np.array([*self.core_indices, self.n_p + 1j * self.k_p])

    def ab(self, n_m=1.42, wavelength=0.532):
        from . import _kernels
        a, _, nmax = _kernels.layered_ab_host([self], float(np.real(n_m)),
                                              float(wavelength))
        return a[0, :nmax[0] + 1]
