'''FP64 restatement of the reference's fitting loop (oracle).

``Optimizer.optimize`` (analysis/Optimizer.py:196-222) hands
``(hologram(p) - data)/noise`` (:257-260) to scipy's
``least_squares(method='lm')`` with the defaults of :102-113; scipy runs
MINPACK ``lmder`` (Moré's trust-region Levenberg-Marquardt) on a
forward-difference Jacobian.  scipy is a third-party dependency that the
reference does not pin (pyproject.toml lists it bare); this container has
scipy 1.18.1.  ``statistics`` restates ``Optimizer._statistics`` (:262-278).

Test infrastructure only: see ``oracle/__init__.py``.
'''
import numpy as np
from scipy.optimize import least_squares
from scipy.linalg import svd
from .field import hologram, aberrated_hologram

PARTICLE_KEYS = ('x_p', 'y_p', 'z_p', 'a_p', 'n_p', 'k_p')
DEFAULT_VARIABLES = ('x_p', 'y_p', 'z_p', 'a_p', 'n_p')
DEFAULT_SETTINGS = {'method': 'lm', 'ftol': 1e-4, 'xtol': 1e-6,
                    'gtol': 1e-6, 'loss': 'linear', 'max_nfev': 2000,
                    'diff_step': 1e-5, 'x_scale': 'jac'}


def statistics(res, npix):
    '''redchi and uncertainties from the final Jacobian by SVD.'''
    ndeg = npix - res.x.size
    redchi = 2. * res.cost / ndeg
    _, s, vt = svd(res.jac, full_matrices=False)
    threshold = np.finfo(float).eps * max(res.jac.shape) * s[0]
    s = s[s > threshold]
    vt = vt[:s.size]
    pcov = np.dot(vt.T / s ** 2, vt)
    return redchi, np.sqrt(redchi * np.diag(pcov))


def fit(data, coordinates, particle, instrument, variables=DEFAULT_VARIABLES,
        settings=None, jac=None, spherical=0.):
    '''One LM fit; returns a dict shaped like ``Optimizer.result``.

    ``data``: (npts,) normalized intensities; ``coordinates``: (2|3, npts);
    ``particle``: dict with the six particle keys (start values), plus
    'fractions' and 'core_indices' for a multilayer sphere whose inner radii
    keep their fractions of the fitted outer radius a_p;
    ``instrument``: dict with n_m, wavelength, magnification, noise.
    ``jac``: optional callable p -> (npts, nvar) dH/dp (not divided by
    noise), standing in for the analytic-Jacobian slot
    (analysis/Optimizer.py:218-220, 251-255).
    ``spherical``: the model is AberratedLorenzMie with this coefficient
    (theory/Aberrated.py:41-85), as when the reference's Optimizer is given
    that model.
    '''
    settings = dict(DEFAULT_SETTINGS if settings is None else settings)
    variables = list(variables)
    noise = instrument.get('noise', 0.05)
    base = dict(particle)

    def params(values):
        p = dict(base)
        p.update(zip(variables, values))
        if 'fractions' in p:  # multilayer: outer radius and index vary
            frac = np.asarray(p['fractions'], dtype=float)
            p['layers'] = (np.append(frac * p['a_p'], p['a_p']),
                           np.append(np.asarray(p['core_indices'], complex),
                                     p['n_p'] + 1j * p.get('k_p', 0.)))
        return p

    def residuals(values):
        if spherical:
            h = aberrated_hologram(coordinates, [params(values)], instrument,
                                   spherical)
        else:
            h = hologram(coordinates, [params(values)], instrument)
        return (h - data) / noise

    if jac is not None:
        settings['jac'] = lambda values: jac(params(values)) / noise
    p0 = np.array([base[v] for v in variables], dtype=float)
    res = least_squares(residuals, p0, **settings)
    redchi, dp = statistics(res, data.size)
    out = {}
    for v, x, d in zip(variables, res.x, dp):
        out[v] = float(x)
        out['d' + v] = float(d)
    out.update(success=bool(res.success), npix=int(data.size),
               redchi=float(redchi), status=int(res.status),
               nfev=int(res.nfev))
    return out
