'''A hologram crop of one particle with its estimator and optimizer (same
contract as analysis/Feature.py).

The crop's Mask excludes saturated (maximum-valued), NaN and infinite
pixels for both the estimator and the optimizer, and keeps the reference's
random-subset fraction (analysis/Feature.py:32-44).  ``optimize`` runs the
device fit of Optimizer; many features are fitted together by
Frame.optimize.
'''
import numpy as np

from ..theory.LorenzMie import LorenzMie
from .Hologram import Hologram
from .Mask import Mask
from .DEEstimator import DEEstimator
from .Optimizer import Optimizer


class Feature(Hologram):
    '''A holographic feature associated with a single particle.'''

    def __init__(self, hologram, model=None, fixed=None):
        # Hologram state copied directly (no recomputation of coordinates)
        self.data = hologram.data
        self.corner = hologram.corner
        self._coordinates = hologram._coordinates
        self._grid = getattr(hologram, 'is_grid', True)
        self.model = model or LorenzMie()
        m = Mask()
        m.shape = self.data.shape
        m.exclude = ((self.data == np.max(self.data)) |
                     np.isnan(self.data) | np.isinf(self.data))
        self.estimator = DEEstimator(model=self.model, exclude=m.exclude)
        self.optimizer = Optimizer(model=self.model, mask=m)
        if fixed is not None:
            self.optimizer.fixed = fixed

    @property
    def mask(self):
        '''Pixel mask shared by the estimator and the optimizer.'''
        return self.optimizer.mask

    @mask.setter
    def mask(self, mask):
        self.estimator.exclude = mask.exclude
        self.optimizer.mask = mask

    @property
    def particle(self):
        return self.model.particle

    @particle.setter
    def particle(self, particle):
        self.model.particle = particle

    @property
    def model(self):
        return self._model

    @model.setter
    def model(self, model):
        self._model = model

    def estimate(self):
        '''Initial parameters by differential evolution (DEEstimator).'''
        return self.estimator.estimate(self)

    def optimize(self):
        '''Fit the crop; a fresh random pixel subset under the mask.'''
        return self.optimizer.optimize(self)

    def predicted(self):
        '''The model's hologram over every pixel of the crop.'''
        self.model.coordinates = self.flat_coordinates
        return self.model.hologram().reshape(self.shape)

    def residuals(self):
        return self.predicted() - self.data
