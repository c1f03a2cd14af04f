'''Oracle tasks for the CPU baseline of bench.py (test infrastructure).

Module-level functions so that a ``spawn`` process pool can run them: one
renders a 201x201 single-sphere hologram with the FP64 oracle plus noise,
the other runs the reference fitting algorithm (scipy least_squares lm with
a forward-difference Jacobian, Optimizer defaults) on it.
'''
import numpy as np

from .field import hologram, meshgrid, DEFAULT_INSTRUMENT
from .fit import fit

KEYS = ('x_p', 'y_p', 'z_p', 'a_p', 'n_p', 'k_p')


def render_201(truth, seed):
    shape = (201, 201)
    rng = np.random.default_rng(seed)
    h = hologram(meshgrid(shape), [dict(zip(KEYS, truth))],
                 DEFAULT_INSTRUMENT)
    return h + rng.normal(0., 0.05, h.shape)


def fit_201(data, start):
    return fit(data, meshgrid((201, 201)), dict(zip(KEYS, start)),
               DEFAULT_INSTRUMENT)


def fit_crop(data, shape, start, fractions=None, core_indices=None,
             settings=None):
    '''The reference fitting algorithm on one crop of any shape; a layered
    sphere keeps its inner radius fractions and indices.  settings: scipy
    least_squares settings (None: the Optimizer's defaults).'''
    particle = dict(zip(KEYS, start))
    if fractions is not None:
        particle['fractions'] = list(fractions)
        particle['core_indices'] = list(core_indices)
    return fit(np.asarray(data).ravel(), meshgrid(tuple(shape)), particle,
               DEFAULT_INSTRUMENT, settings=settings)
