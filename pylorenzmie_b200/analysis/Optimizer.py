'''Drop-in Optimizer whose Levenberg-Marquardt loop runs on the GPU.

Same constructor, settings, ``fixed``/``variables``, ``result``,
``metadata`` and ``report()`` as analysis/Optimizer.py.  ``optimize``
returns the same pandas Series (:166-186).  With the default settings
(method 'lm', linear loss, x_scale 'jac') and free variables among the
sphere's x_p, y_p, z_p, a_p, n_p, k_p, the whole fit -- residuals,
analytic Jacobian, J^T J reduction, MINPACK's damped step and its
convergence tests -- runs on the device in one call (``lmb_fit_batch``;
``lmb_fit_batch_layered`` for LayeredSphere particles,
``lmb_fit_batch_aberrated`` for an AberratedLorenzMie model whose
``spherical`` is fixed).  Other settings (robust losses, 'trf'/'dogbox',
explicit x_scale, instrument parameters or ``spherical`` as variables) keep
the reference's host loop:
scipy.optimize.least_squares calling this model's GPU ``hologram()`` and,
when every variable is covered, its analytic ``jac()``.

``optimize_batch`` fits many features in one device call and returns a
DataFrame with one ``result``-shaped row per feature (the batched form of
Frame.optimize, analysis/Frame.py:163-174).
'''
import numpy as np
import pandas as pd
from scipy.linalg import svd
from scipy.optimize import least_squares

from ..lib import LMObject
from ..theory.LorenzMie import LorenzMie
from .Hologram import Hologram
from .Mask import Mask
from . import _fit

PARAM_KEYS = _fit.PARAM_KEYS


class _Result:
    '''Final state of one fit (the fields Optimizer.result needs).'''

    def __init__(self, x, success, redchi, dp, status, nfev, cost, jac=None):
        self.x = np.asarray(x, dtype=float)
        self.success = bool(success)
        self.redchi = float(redchi)
        self.dp = np.asarray(dp, dtype=float)
        self.status = int(status)
        self.nfev = int(nfev)
        self.cost = float(cost)
        self.jac = jac


class Optimizer(LMObject):
    '''Fit a Lorenz-Mie model to holographic data.'''

    method: str = 'b200'

    def __init__(self, model=None, mask=None, robust=False, fixed=None,
                 settings=None, **kwargs):
        self.model = model or LorenzMie(**kwargs)
        if self.method not in self.model.method:
            raise TypeError('Model not compatible with Optimizer')
        self.mask = mask
        self.settings = settings
        default_fixed = ('wavelength magnification numerical_aperture '
                         'n_m noise k_p').split()
        self.fixed = fixed if fixed is not None else default_fixed
        self.robust = robust
        self._data = None
        self._result = None

    @property
    def properties(self):
        return dict(settings=self.settings, fixed=self.fixed)

    @properties.setter
    def properties(self, properties):
        for name, value in properties.items():
            if hasattr(self, name):
                setattr(self, name, value)

    @property
    def settings(self):
        return self._settings

    @settings.setter
    def settings(self, settings):
        if settings is None:
            settings = dict(_fit.DEFAULT_SETTINGS)
        self._settings = settings

    @property
    def robust(self):
        return self.settings['loss'] != 'linear'

    @robust.setter
    def robust(self, robust):
        if robust:
            self.settings['method'] = 'trf'
            self.settings['loss'] = 'cauchy'
        else:
            self.settings['method'] = 'lm'
            self.settings['loss'] = 'linear'

    @property
    def fraction(self):
        return 1.0 if self.mask is None else self.mask.fraction

    @fraction.setter
    def fraction(self, fraction):
        if self.mask is None:
            self.mask = Mask()
        self.mask.fraction = fraction

    @property
    def fixed(self):
        return self._fixed

    @fixed.setter
    def fixed(self, fixed):
        self._fixed = list(fixed)
        self._variables = [p for p in self.model.properties if p not in fixed]

    @property
    def variables(self):
        return self._variables

    @variables.setter
    def variables(self, variables):
        self._variables = list(variables)
        self._fixed = [p for p in self.model.properties if p not in variables]

    @property
    def result(self):
        if self._result is None:
            return None
        a = self.variables
        b = ['d' + v for v in a]
        keys = list(sum(zip(a, b), ()))
        keys.extend('success npix redchi'.split())
        values = list(sum(zip(self._result.x, self._result.dp), ()))
        values.extend([self._result.success, self._data.size,
                       self._result.redchi])
        return pd.Series(dict(zip(keys, values)))

    @property
    def metadata(self):
        metadata = {key: self.model.properties[key] for key in self.fixed
                    if key in self.model.properties}
        metadata.update(self.settings)
        return pd.Series(metadata)

    # ------------------------------------------------------------------
    def _device_fit_ok(self):
        s = self.settings
        if s.get('method', 'lm') != 'lm' or s.get('loss', 'linear') != 'linear':
            return False
        xs = s.get('x_scale', 'jac')
        if not (isinstance(xs, str) and xs == 'jac'):
            return False
        if any(key in s for key in ('jac', 'bounds', 'callback', 'args',
                                    'kwargs')):
            return False
        if not set(self.variables) <= set(PARAM_KEYS) or not self.variables:
            return False
        p = self.model.particle
        return len(p) == 1 and hasattr(p, 'a_p')

    def _pixels(self, hologram):
        '''(data, grid, coords) of a hologram under this optimizer's mask.'''
        if self.mask is None:
            data = hologram.flat_data
            if getattr(hologram, 'is_grid', False):
                ny, nx = hologram.shape
                grid = (float(hologram.corner[0]), float(hologram.corner[1]),
                        ny, nx)
                return data, grid, hologram.flat_coordinates
            return data, None, hologram.flat_coordinates
        data, coords = self.mask.apply(hologram)
        return data, None, coords

    def optimize(self, hologram):
        '''Fit the model to ``hologram``; returns the result Series.'''
        data, grid, coords = self._pixels(hologram)
        self._data = np.asarray(data)
        self.model.coordinates = coords
        if self._device_fit_ok():
            self._optimize_device(data, grid, coords)
        else:
            self._optimize_host()
        return self.result

    def _start(self):
        '''(1, 6) start vector of the model's single sphere.'''
        part = self.model.particle[0] if len(self.model.particle) else None
        r = np.asarray(part.r_p, float) + np.asarray(
            getattr(part, 'r_0', (0., 0., 0.)), float)
        return np.array([[r[0], r[1], r[2], part.a_p, part.n_p,
                          getattr(part, 'k_p', 0.)]])

    def _aberration(self):
        '''Spherical-aberration coefficient c of the model (0: ideal
        optics; AberratedLorenzMie models carry the phase of
        theory/Aberrated.py into the device fit).'''
        return float(getattr(self.model, '_aberration', lambda: 0.)())

    def _optimize_device(self, data, grid, coords):
        packed = _fit.PackedFeatures([(data, grid, coords)])
        part = self.model.particle[0] if len(self.model.particle) else None
        params, res = _fit.fit_packed(packed, self._start(),
                                      self.model.instrument,
                                      self.variables, self.settings,
                                      device=self.model.device,
                                      layers=_fit.layers_of([part]),
                                      aberration=self._aberration())
        status = int(res['status'][0])
        if status == -1:
            raise ValueError("Method 'lm' doesn't work when the number of "
                             'residuals is less than the number of variables.')
        if status == -2:
            raise ValueError('Residuals are not finite in the initial point.')
        self._accept(params[0], res[0])

    def _accept(self, fitted, res):
        '''Take a device fit's result: the model is left at the fitted
        values (as scipy leaves it at its last evaluation) and ``result``
        reports them.'''
        part = self.model.particle[0] if len(self.model.particle) else None
        idx = [PARAM_KEYS.index(v) for v in self.variables]
        r0 = np.asarray(getattr(part, 'r_0', (0., 0., 0.)), float)
        self.model.properties = {v: float(fitted[PARAM_KEYS.index(v)] -
                                          (r0[PARAM_KEYS.index(v)] if
                                           PARAM_KEYS.index(v) < 3 else 0.))
                                 for v in self.variables}
        self._result = _Result(fitted[idx], res['success'], res['redchi'],
                               res['dparams'][idx], int(res['status']),
                               res['nfev'], res['cost'])

    def _optimize_host(self):
        p0 = np.array([self.model.properties[p] for p in self.variables])
        settings = dict(self.settings)
        jac_params = getattr(self.model, 'jac_params', None)
        if jac_params is not None and set(self.variables) <= jac_params:
            settings['jac'] = self._analytical_jac
        res = least_squares(self._residuals, p0, **settings)
        redchi, dp = self._statistics(res)
        self._result = _Result(res.x, res.success, redchi, dp, res.status,
                               res.nfev, res.cost, res.jac)

    def _analytical_jac(self, values):
        self.model.properties = dict(zip(self.variables, values))
        J = self.model.jac()
        noise = self.model.instrument.noise
        return np.column_stack([J[p] for p in self.variables]) / noise

    def _residuals(self, values):
        self.model.properties = dict(zip(self.variables, values))
        noise = self.model.instrument.noise
        return (self.model.hologram() - self._data) / noise

    def _statistics(self, res):
        ndeg = self._data.size - res.x.size
        redchi = 2. * res.cost / ndeg
        _, s, VT = svd(res.jac, full_matrices=False)
        threshold = np.finfo(float).eps * max(res.jac.shape) * s[0]
        s = s[s > threshold]
        VT = VT[:s.size]
        pcov = np.dot(VT.T / s ** 2, VT)
        return redchi, np.sqrt(redchi * np.diag(pcov))

    def report(self):
        result = self.result
        if result is None:
            raise RuntimeError('optimize() must be called before report()')
        units = {'x_p': 'pixels', 'y_p': 'pixels', 'z_p': 'pixels',
                 'a_p': 'μm'}
        fmt = {'x_p': '.2f', 'y_p': '.2f', 'z_p': '.2f', 'a_p': '.3f'}
        lines = []
        for p in self.variables:
            f = fmt.get(p, '.4f')
            suffix = f' {units[p]}' if p in units else ''
            lines.append(f"{p} = {result[p]:{f}} ± {result['d' + p]:{f}}"
                         f'{suffix}')
        lines += [f'npixels = {result.npix:.0f}',
                  f'χ² = {result.redchi:.2f}']
        return '\n'.join(lines)

    # ------------------------------------------------------------------
    def optimize_batch(self, holograms, particles=None, starts=None,
                       autotune=None, chunks=None):
        '''Fit one sphere per hologram, all on the device in one call.

        holograms : list of Hologram (crops; any sizes)
        particles : list of Sphere (or LayeredSphere, one layer count)
                    start values; the layer structure of layered spheres
                    is kept, their outer radius and index are fitted
        starts    : array (B, 6) of x_p, y_p, z_p, a_p, n_p, k_p (overrides
                    the particles' start values)
        autotune  : time the evaluation kernel's launch shapes once per
                    problem class and use the fastest (default: batches of
                    64 features or more)
        chunks    : pipeline depth: the batch is fitted in this many parts,
                    each on its own stream, so that converting and copying
                    one part overlaps the fit of the previous one (default:
                    1 below ~2 Mpx, up to 4 above)
        Returns a DataFrame, one row per feature, with the columns of
        ``result`` plus ``status`` and ``nfev``.
        '''
        if not self._device_fit_ok() and not (
                set(self.variables) <= set(PARAM_KEYS)):
            raise ValueError('optimize_batch fits sphere parameters only')
        layers = None
        if particles is not None:
            layers = _fit.layers_of(list(particles))
        if starts is None:
            if particles is None:
                raise ValueError('give particles or starts')
            starts = np.array([[*(np.asarray(p.r_p, float) + np.asarray(
                getattr(p, 'r_0', (0., 0., 0.)), float)), p.a_p, p.n_p,
                getattr(p, 'k_p', 0.)] for p in particles], dtype=float)
        items = [self._pixels(h) for h in holograms]
        if autotune is None:
            autotune = len(holograms) >= 64
        params, res, npix = _fit.fit_items(
            items, starts, self.model.instrument, self.variables,
            self.settings, device=self.model.device, layers=layers,
            autotune=autotune, chunks=chunks, aberration=self._aberration())
        return batch_frame(params, res, npix, self.variables)


    def optimize_stream(self, batches, autotune=None, depth=None):
        '''Fit a stream of batches (video frames, say), pipelined: while
        the GPU fits one batch, the next is converted and copied.  Yields
        one DataFrame per batch, in order, as optimize_batch returns it.

        batches : iterable of (holograms, starts) or (holograms,
                  particles) pairs; starts an array (B, 6), particles a
                  list of Sphere or LayeredSphere start values
        autotune: time the evaluation kernel's launch shapes on the first
                  batch (default: when it has 64 features or more)
        depth   : fits running at once; the next batch is converted and
                  copied while they run.  Default 2, which keeps the GPU
                  busy; 4 when the first batch holds LayeredSphere
                  particles, whose batches end with long single-fit tails
                  that further fits fill
        '''
        if not self._device_fit_ok() and not (
                set(self.variables) <= set(PARAM_KEYS)):
            raise ValueError('optimize_stream fits sphere parameters only')
        variables = list(self.variables)
        first = [True]

        def items():
            for holograms, second in batches:
                layers = None
                if not (len(second) and hasattr(second[0], 'r_p')):
                    starts = np.asarray(second, dtype=float).reshape(-1, 6)
                else:
                    layers = _fit.layers_of(list(second))
                    starts = np.array([[*(np.asarray(p.r_p, float) +
                                          np.asarray(getattr(
                                              p, 'r_0', (0., 0., 0.)),
                                              float)), p.a_p, p.n_p,
                                        getattr(p, 'k_p', 0.)]
                                       for p in second], dtype=float)
                if first[0]:
                    first[0] = False
                    self._stream_tune = (autotune if autotune is not None
                                         else len(holograms) >= 64)
                yield [self._pixels(h) for h in holograms], starts, layers

        gen = items()
        # the first batch decides autotuning before the pipeline starts
        try:
            head = next(gen)
        except StopIteration:
            return

        def chain():
            yield head
            yield from gen
        if depth is None:
            depth = 2 if head[2] is None else 4
        for params, res, npix in _fit.fit_stream(
                chain(), self.model.instrument, variables, self.settings,
                device=self.model.device, autotune=self._stream_tune,
                depth=depth, aberration=self._aberration()):
            yield batch_frame(params, res, npix, variables)


def batch_frame(params, res, npix, variables):
    '''DataFrame of batched fit results in the Optimizer.result layout.'''
    idx = [PARAM_KEYS.index(v) for v in variables]
    cols = {}
    for v, j in zip(variables, idx):
        cols[v] = params[:, j]
        cols['d' + v] = res['dparams'][:, j]
    cols['success'] = res['success'].astype(bool)
    cols['npix'] = np.asarray(npix)
    cols['redchi'] = res['redchi']
    cols['status'] = res['status']
    cols['nfev'] = res['nfev']
    return pd.DataFrame(cols)
