'''Normalized hologram with pixel coordinates (same contract as
analysis/Hologram.py): flat views and coordinate-aware crops.'''
from dataclasses import dataclass

import numpy as np

from ..lib import meshgrid


@dataclass(eq=False)
class Hologram:
    data: np.ndarray
    corner: tuple = (0., 0.)

    def __post_init__(self):
        self._coordinates = meshgrid(self.data.shape, corner=self.corner,
                                     flatten=False)

    def __eq__(self, other):
        if not isinstance(other, Hologram):
            return NotImplemented
        return (np.array_equal(self.data, other.data) and
                self.corner == other.corner)

    @property
    def shape(self):
        return self.data.shape

    @property
    def coordinates(self):
        return self._coordinates

    @property
    def flat_data(self):
        return self.data.ravel()

    @property
    def flat_coordinates(self):
        return self._coordinates.reshape(2, -1)

    @property
    def is_grid(self):
        '''True when the coordinates are the unit-step grid at ``corner``
        (then the fit kernel regenerates them instead of reading them).'''
        return getattr(self, '_grid', True)

    @staticmethod
    def _from_slice(data, coordinates):
        h = object.__new__(Hologram)
        h.data = data
        h.corner = (float(coordinates[0, 0, 0]), float(coordinates[1, 0, 0]))
        h._coordinates = coordinates
        ny, nx = data.shape
        g = meshgrid((ny, nx), corner=h.corner, flatten=False)
        h._grid = bool(np.array_equal(g, coordinates))
        return h

    def __getitem__(self, key):
        sy, sx = key
        return Hologram._from_slice(self.data[key],
                                    self._coordinates[:, sy, sx])
