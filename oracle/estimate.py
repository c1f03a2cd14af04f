'''FP64 restatement of the reference's global estimators (oracle).

``de_estimate`` follows DEEstimator.estimate (analysis/DEEstimator.py:
127-169): x_p, y_p pinned to the coordinate means (:140-141); a random
pixel subset drawn from numpy's global RNG as Mask does
(analysis/Mask.py:64-72, 74-80, 82-105: rand(*shape) < fraction, excluded
pixels removed); objective sum(((H - data)/noise)^2) with NaN skipped
(:32-37); scipy's differential_evolution over the bounds (:153-166) with
the reference's settings (:103-106).  ``radial_estimate`` follows
RadialEstimator.estimate (analysis/RadialEstimator.py:122-170): azimuthal
average about the pinned position (lib/Azimuthal.py:avg: integer-radius
bins) compared with the model along (x_p + r, y_p).  scipy is the
unpinned third-party dependency named in oracle/fit.py.

Test infrastructure only: see ``oracle/__init__.py``.
'''
import numpy as np
from scipy.optimize import differential_evolution

from .field import hologram

DEFAULT_BOUNDS = {'z_p': (10., 600.), 'a_p': (0.25, 10.0), 'n_p': (1.0, 3.0)}
SETTINGS = {'tol': 0.01, 'polish': False, 'updating': 'deferred'}


def _search(data, coords, particle, instrument, bounds, popsize, seed):
    variables = list(bounds)
    noise = instrument.get('noise', 0.05)

    def objective(values):
        p = dict(particle)
        p.update(zip(variables, values))
        with np.errstate(over='ignore', invalid='ignore'):
            diff = (hologram(coords, [p], instrument) - data) / noise
            return float(np.nansum(diff ** 2))
    with np.errstate(over='ignore', invalid='ignore'):
        res = differential_evolution(objective, list(bounds.values()),
                                     popsize=popsize, seed=seed, workers=1,
                                     **SETTINGS)
    out = dict(particle)
    out.update(zip(variables, res.x))
    return out, res


def de_estimate(data, coordinates, particle, instrument,
                bounds=DEFAULT_BOUNDS, fraction=0.02, exclude=None,
                popsize=10, seed=None):
    '''data (ny, nx); coordinates (2, ny, nx); particle dict (start values
    of the fixed parameters).  Draws the pixel subset from numpy's global
    RNG; returns (particle dict at the estimate, OptimizeResult).'''
    p = dict(particle)
    p['x_p'] = float(coordinates[0].mean())
    p['y_p'] = float(coordinates[1].mean())
    mask = np.random.rand(*data.shape) < fraction
    if exclude is not None and exclude.shape == mask.shape:
        mask[exclude] = False
    return _search(data[mask], coordinates[:, mask], p, instrument, bounds,
                   popsize, seed)


def azimuthal_avg(data, center):
    '''Mean of the pixels in each integer-radius bin about center (x, y).'''
    ny, nx = data.shape
    r = np.hypot.outer(np.arange(ny) - center[1],
                       np.arange(nx) - center[0]).astype(np.int32).ravel()
    return np.bincount(r, data.ravel()) / np.bincount(r)


def radial_estimate(data, coordinates, corner, particle, instrument,
                    bounds=DEFAULT_BOUNDS, popsize=10, seed=None):
    p = dict(particle)
    x_p = float(coordinates[0].mean())
    y_p = float(coordinates[1].mean())
    p['x_p'], p['y_p'] = x_p, y_p
    profile = azimuthal_avg(data, (x_p - corner[0], y_p - corner[1]))
    radii = np.arange(len(profile), dtype=float)
    coords = np.vstack([x_p + radii, np.full(len(profile), y_p)])
    return _search(profile, coords, p, instrument, bounds, popsize, seed)
