'''Random pixel subset for fitting (same contract as analysis/Mask.py).'''
from dataclasses import dataclass

import numpy as np

from ..lib import LMObject


@dataclass
class Mask(LMObject):
    shape: tuple | None = None
    fraction: float = 0.1
    exclude: np.ndarray | None = None

    def __post_init__(self):
        self._mask = np.empty((0, 0), dtype=bool)
        self.update()

    def __setattr__(self, prop, value):
        super().__setattr__(prop, value)
        if prop in ('shape', 'fraction', 'exclude') and hasattr(self, '_mask'):
            self.update()

    def __call__(self):
        return self._mask

    @LMObject.properties.getter
    def properties(self):
        return dict(fraction=self.fraction)

    def _select(self):
        if self.shape is None:
            return
        self._mask = np.random.rand(*self.shape) < self.fraction

    def update(self):
        if self.shape is None:
            return
        self._select()
        if self.exclude is not None and self.exclude.shape == self._mask.shape:
            self._mask[self.exclude] = False

    def apply(self, hologram):
        '''Selected pixel values (nsel,) and coordinates (2, nsel); a fresh
        random subset each call (analysis/Mask.py:82-105).'''
        self.shape = hologram.shape
        m = self._mask
        return hologram.data[m], hologram.coordinates[:, m]
