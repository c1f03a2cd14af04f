'''Homogeneous sphere (same contract as theory/Sphere.py).

``ab`` / ``mie_coefficients`` run the FP64 coefficient kernel of the CUDA
library (``lmb_sphere_ab``) and return numpy complex128 (nmax+1, 2).
'''
from dataclasses import dataclass

import numpy as np

from .Particle import Particle
from ..lib import LMObject


@dataclass
class Sphere(Particle):
    a_p: float = 1.
    n_p: float = 1.5
    k_p: float = 0.

    @property
    def d_p(self):
        return 2. * self.a_p

    @d_p.setter
    def d_p(self, d_p):
        self.a_p = d_p / 2.

    @LMObject.properties.getter
    def properties(self):
        return {**Particle.properties.fget(self),
                'a_p': self.a_p, 'n_p': self.n_p, 'k_p': self.k_p}

    def ab(self, n_m=1.42, wavelength=0.532):
        return Sphere.mie_coefficients(self.a_p, self.n_p, self.k_p, n_m,
                                       wavelength)

    @staticmethod
    def wiscombe_yang(x, m):
        '''Number of partial waves (theory/Sphere.py:91-123), host side;
        the kernels evaluate the same rule on the device.'''
        x = np.atleast_1d(np.asarray(x, dtype=float))
        m = np.atleast_1d(np.asarray(m, dtype=complex))
        xl = abs(x[-1])
        if xl <= 8.:
            ns = np.floor(xl + 4. * np.cbrt(xl) + 1.)
        elif xl <= 4200.:
            ns = np.floor(xl + 4.05 * np.cbrt(xl) + 2.)
        else:
            ns = np.floor(xl + 4. * np.cbrt(xl) + 2.)
        xm = np.abs(x * m)
        xm_1 = np.abs(np.roll(x, -1) * m)
        return int(max(ns, xm.max(), xm_1.max()))

    @staticmethod
    def neves_pisignano(x, precision=6.):
        return int(x + 0.76 * np.cbrt(precision * precision * x) - 4.1)

    @staticmethod
    def mie_coefficients(a_p, n_p, k_p, n_m, wavelength):
        from . import _kernels
        rec = np.zeros(1, dtype=_kernels.SPHERE_DTYPE)
        rec['a_p'], rec['n_p'], rec['k_p'] = a_p, n_p, k_p
        ab, _, nmax = _kernels.sphere_ab_host(rec, float(np.real(n_m)),
                                              float(wavelength))
        return ab[0, :nmax[0] + 1]
