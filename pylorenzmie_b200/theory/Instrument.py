'''Microscope optics (same contract as theory/Instrument.py).'''
from dataclasses import dataclass

import numpy as np

from ..lib import LMObject


@dataclass
class Instrument(LMObject):
    wavelength: float = 0.447
    magnification: float = 0.048
    numerical_aperture: float = 1.45
    noise: float = 0.05
    n_m: float = 1.340

    @LMObject.properties.getter
    def properties(self):
        return {'n_m': self.n_m,
                'wavelength': self.wavelength,
                'magnification': self.magnification,
                'numerical_aperture': self.numerical_aperture,
                'noise': self.noise}

    def wavenumber(self, in_medium=True, scaled=True):
        '''Wave number; rad/pixel by default (theory/Instrument.py:46-70).'''
        k = 2. * np.pi / self.wavelength
        if in_medium:
            k *= self.n_m
        if scaled:
            k *= self.magnification
        return k
