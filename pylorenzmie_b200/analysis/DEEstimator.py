'''Global estimate of a sphere's parameters by differential evolution, with
each generation's population evaluated on the GPU in one launch.

Same fields, defaults and behaviour as analysis/DEEstimator.py: x_p, y_p
are pinned to the crop's coordinate means (:140-141), a fresh random
subset of ``fraction`` of the pixels (minus ``exclude``) is drawn once per
call (:143-146), and scipy's differential_evolution minimizes
sum(((H - data)/noise)^2) with NaN residuals skipped (:32-37) over
``bounds`` (:153-166).  The reference evaluates each candidate with one
model.hologram() call, spread over worker processes; here a generation is
one lmb_chi2_batch launch, and the search is scipy's algorithm with
``updating='deferred'`` (the reference's setting) either as run_populations
restates it (the estimators' settings; no per-candidate Python) or as
scipy itself with ``vectorized=True``.  With the same seed and an FP64
model the search follows the reference's trajectory; with FP32 sums the
energies differ by rounding only.  run_searches / estimate_many search many
features together, one lmb_chi2_crops launch per generation of all of them.
'''
from dataclasses import dataclass, field

import numpy as np
import pandas as pd
from scipy.optimize import differential_evolution

from .BaseEstimator import BaseEstimator
from .Mask import Mask
from ._de import run_populations, supported
from ._device_de import device_searches
from ._population import (CropPopulations, PopulationChi2, aberration,
                          batchable, de_settings, lockstep_de)

DEFAULT_BOUNDS = {
    'z_p': (10., 600.),
    'a_p': (0.25, 10.0),
    'n_p': (1.0, 3.0),
}


class _HostObjective:
    '''One model.hologram() per candidate: for searches over variables the
    population kernel does not cover (instrument properties, layered or
    multi-particle models).'''

    def __init__(self, model, data, variables, noise):
        self.model, self.data = model, data
        self.variables, self.noise = variables, noise

    def __call__(self, x):
        x = np.asarray(x, dtype=float)
        X = x.reshape(len(self.variables), -1)
        out = np.empty(X.shape[1])
        for s in range(X.shape[1]):
            self.model.properties = dict(zip(self.variables, X[:, s]))
            with np.errstate(over='ignore', invalid='ignore'):
                diff = (self.model.hologram() - self.data) / self.noise
                out[s] = float(np.nansum(diff ** 2))
        return float(out[0]) if x.ndim == 1 else out


def run_search(model, data, coords, variables, bounds, noise, popsize, seed,
               settings, device_search=False):
    '''scipy differential_evolution over ``variables`` with the population
    objective; returns the OptimizeResult.  The model's coordinates are
    restored on exit.  ``device_search``: the whole search on the GPU
    (device_searches), where the model and settings allow it.'''
    if device_search and batchable(model, variables) and supported(settings):
        return device_searches([dict(
            model=model, data=data, coords=coords, variables=variables,
            bounds=bounds, noise=noise, popsize=popsize, seed=seed,
            settings=settings)])[0]
    saved = model.coordinates
    try:
        if batchable(model, variables):
            if supported(settings):
                # the crops objective over this one crop: the same values
                # as PopulationChi2, with its buffers kept between
                # generations
                pop = CropPopulations([(model, data, coords, variables)],
                                      noise)
                problem = dict(bounds=bounds, popsize=popsize, seed=seed,
                               settings=settings)
                with np.errstate(over='ignore', invalid='ignore'):
                    return run_populations([problem], pop.evaluate)[0]
            objective = PopulationChi2(model, data, coords, variables, noise)
        else:
            model.coordinates = coords
            objective = _HostObjective(model, data, variables, noise)
        with np.errstate(over='ignore', invalid='ignore'):
            return differential_evolution(objective, bounds, popsize=popsize,
                                          seed=seed, **de_settings(settings))
    finally:
        model.coordinates = saved


def run_searches(searches, workers=256):
    '''run_search for each of ``searches`` (dicts of its arguments); returns
    the OptimizeResults in order.  Searches whose models share the device,
    the instrument, the noise and the precision run side by side, every
    generation of all of them in one lmb_chi2_crops launch (run_populations,
    or scipy on threads in lockstep_de for settings that form does not
    cover); the rest one at a time.  Each result is the one run_search
    gives.'''
    import torch
    results = [None] * len(searches)
    groups = {}
    for i, sr in enumerate(searches):
        m = sr['model']
        if not batchable(m, sr['variables']):
            groups.setdefault(None, []).append(i)
            continue
        inst = m.instrument
        key = (str(m.device), float(inst.n_m), float(inst.wavelength),
               float(inst.magnification), float(sr['noise']),
               bool(getattr(m, 'double_precision', False)), aberration(m))
        if sr.get('device_search') and supported(sr['settings']):
            # one device loop: the same variables, population and mutation
            st = sr['settings'] or {}
            key = key + ('device', tuple(sr['variables']), sr['popsize'],
                         repr(st.get('mutation', (0.5, 1))))
        groups.setdefault(key, []).append(i)
    for key, idx in groups.items():
        if key is not None and 'device' in key:
            out = device_searches([searches[i] for i in idx])
            for i, r in zip(idx, out):
                results[i] = r
            continue
        if key is None or len(idx) == 1:
            for i in idx:
                results[i] = run_search(**searches[i])
            continue
        members = [searches[i] for i in idx]
        pop = CropPopulations([(sr['model'], sr['data'], sr['coords'],
                                sr['variables']) for sr in members],
                              members[0]['noise'])
        if all(supported(sr['settings']) for sr in members):
            with np.errstate(over='ignore', invalid='ignore'):
                out = run_populations(members, pop.evaluate)
        else:
            dev = pop.device
            out = lockstep_de(members, pop.evaluate, workers, dev,
                              torch.cuda.current_stream(dev))
        for i, r in zip(idx, out):
            results[i] = r
    return results


def estimate_many(estimators, holograms, series=True):
    '''estimator.estimate(hologram) for each pair, the searches side by
    side (run_searches); returns the Series in order (with
    ``series=False`` only the models are left at the estimates, and the
    result is None).  Estimators that share a model run one after another,
    as the model carries each search's start.'''
    estimators, holograms = list(estimators), list(holograms)
    if len({id(e.model) for e in estimators}) < len(estimators):
        out = [e.estimate(h) for e, h in zip(estimators, holograms)]
        return out if series else None
    searches = [e.search(h) for e, h in zip(estimators, holograms)]
    results = run_searches(searches)
    out = [e.accept(sr, r, series=series)
           for e, sr, r in zip(estimators, searches, results)]
    return out if series else None


@dataclass
class DEEstimator(BaseEstimator):
    '''Estimate initial particle parameters by global search.'''

    model: object
    bounds: dict = field(default_factory=lambda: DEFAULT_BOUNDS.copy())
    fraction: float = 0.02
    exclude: np.ndarray | None = None
    popsize: int = 10
    seed: int | None = None
    settings: dict = field(default_factory=lambda: {'tol': 0.01,
                                                     'polish': False,
                                                     'updating': 'deferred',
                                                     'workers': -1})
    device_search: bool = False   # the whole search on the GPU

    @property
    def properties(self):
        return dict(fraction=self.fraction, popsize=self.popsize,
                    bounds=self.bounds, settings=self.settings)

    @properties.setter
    def properties(self, properties):
        for name, value in properties.items():
            if hasattr(self, name):
                setattr(self, name, value)

    def search(self, hologram):
        '''The arguments of run_search for this hologram: x_p, y_p pinned
        to the crop's centre and a fresh random pixel subset drawn
        (analysis/DEEstimator.py:146-156).'''
        self.model.particle.x_p = float(hologram.coordinates[0].mean())
        self.model.particle.y_p = float(hologram.coordinates[1].mean())
        mask = Mask(fraction=self.fraction)
        if self.exclude is not None:
            mask.exclude = self.exclude
        data, coords = mask.apply(hologram)
        return dict(model=self.model, data=data, coords=coords,
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
        '''Estimate particle parameters; returns the particle's properties
        as a pandas Series and leaves the model at the estimate.'''
        search = self.search(hologram)
        return self.accept(search, run_search(**search))
