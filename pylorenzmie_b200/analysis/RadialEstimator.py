'''Global estimate from the azimuthal profile, population on the GPU.

Same fields, defaults and behaviour as analysis/RadialEstimator.py: x_p,
y_p pinned to the crop's coordinate means, the azimuthal average of the
crop about them (lib/Azimuthal.avg) compared with the model along the
radial spoke (x_p + r, y_p), r = 0, 1, ..., by scipy's
differential_evolution over ``bounds``; each generation's population is one
lmb_chi2_batch launch (see DEEstimator).
'''
from dataclasses import dataclass, field

import numpy as np
import pandas as pd

from ..lib import Azimuthal
from .BaseEstimator import BaseEstimator
from .DEEstimator import DEFAULT_BOUNDS, run_search


@dataclass
class RadialEstimator(BaseEstimator):
    '''Estimate particle parameters by global search on the radial profile.'''

    model: object
    bounds: dict = field(default_factory=lambda: DEFAULT_BOUNDS.copy())
    popsize: int = 10
    seed: int | None = None
    settings: dict = field(default_factory=lambda: {'tol': 0.01,
                                                     'polish': False,
                                                     'updating': 'deferred',
                                                     'workers': 1})
    device_search: bool = False   # the whole search on the GPU

    @property
    def properties(self):
        return dict(popsize=self.popsize, bounds=self.bounds,
                    settings=self.settings)

    @properties.setter
    def properties(self, properties):
        for name, value in properties.items():
            if hasattr(self, name):
                setattr(self, name, value)

    def search(self, hologram):
        '''The arguments of run_search for this hologram: the azimuthal
        profile about the crop's centre along the radial spoke
        (analysis/RadialEstimator.py:134-147).'''
        x_p = float(hologram.coordinates[0].mean())
        y_p = float(hologram.coordinates[1].mean())
        self.model.particle.x_p = x_p
        self.model.particle.y_p = y_p
        cx, cy = hologram.corner
        profile = Azimuthal.avg(hologram.data, center=(x_p - cx, y_p - cy))
        radii = np.arange(len(profile), dtype=float)
        coords = np.vstack([x_p + radii, np.full(len(profile), y_p)])
        return dict(model=self.model, data=profile, coords=coords,
                    variables=list(self.bounds.keys()),
                    bounds=list(self.bounds.values()),
                    noise=self.model.instrument.noise, popsize=self.popsize,
                    seed=self.seed, settings=self.settings,
                    device_search=self.device_search)

    def accept(self, search, result, series=True):
        '''Leave the model at the search's result; its properties as a
        Series (None with ``series=False``, for callers that keep only the
        model state).'''
        self.model.properties = dict(zip(search['variables'], result.x))
        if series:
            return pd.Series(self.model.particle.properties)

    def estimate(self, hologram):
        search = self.search(hologram)
        return self.accept(search, run_search(**search))
