'''Many differential-evolution searches stepped together, without threads.

scipy.optimize.differential_evolution (the search of the reference's
DEEstimator and RadialEstimator, analysis/DEEstimator.py:158-166,
analysis/RadialEstimator.py:150-158) spends most of its time per generation
in per-candidate Python.  ``run_populations`` advances every search of a
frame a generation at a time and hands all their candidates to one
evaluation (one lmb_chi2_crops launch).

Each search follows scipy 1.18's algorithm for the settings the estimators
use (strategy 'best1bin', init 'latinhypercube', updating 'deferred',
dithered mutation, no polish, constraints or integrality): the same
population arithmetic, and the same calls on the search's own random
generator in the same order (the latin-hypercube draw and one permutation
per parameter; per generation the dither draw, one shuffle of the kept
index permutation per candidate, the fill points, the crossover draws and
the redraw of out-of-bounds trial parameters).  A seeded search therefore
returns exactly what differential_evolution returns for it; searches that
draw from numpy's global generator (seed None) interleave their draws, so
each is a valid search but not the one a lone call would make.
``supported`` tells which settings this covers; the estimators run the rest
through scipy.
'''
import ctypes
import numbers

import numpy as np
from scipy.optimize import OptimizeResult

from .. import _native

_SUCCESS = 'Optimization terminated successfully.'
_MAXITER = 'Maximum number of iterations has been exceeded.'

# settings this form follows exactly (anything else goes to scipy)
_DEFAULTS = dict(strategy='best1bin', maxiter=1000, tol=0.01,
                 mutation=(0.5, 1), recombination=0.7, polish=True,
                 init='latinhypercube', atol=0, updating='immediate',
                 workers=1, vectorized=False, disp=False, callback=None,
                 x0=None, constraints=(), integrality=None, args=())


def supported(settings):
    '''True when ``settings`` (differential_evolution keywords besides
    bounds, popsize and seed) are ones this form reproduces.'''
    s = dict(settings)
    for key in s:
        if key not in _DEFAULTS:
            return False
    get = lambda k: s.get(k, _DEFAULTS[k])
    if get('strategy') != 'best1bin' or get('init') != 'latinhypercube':
        return False
    if get('polish') or get('disp') or get('callback') is not None:
        return False
    if get('x0') is not None or get('integrality') is not None:
        return False
    if get('constraints') not in ((), [], None) or get('args') not in ((), []):
        return False
    maxiter = get('maxiter')
    if maxiter is not None and (not isinstance(maxiter, numbers.Integral)
                                or maxiter < 1):
        return False
    m = get('mutation')
    m = np.atleast_1d(np.asarray(m, dtype=float))
    if m.size not in (1, 2) or not np.all(np.isfinite(m)) or \
            np.any(m >= 2) or np.any(m < 0):
        return False
    return True


def _generator(seed):
    '''The search's random generator, as scipy's check_random_state.'''
    if seed is None or seed is np.random:
        return np.random.mtrand._rand
    if isinstance(seed, (numbers.Integral, np.integer)):
        return np.random.RandomState(seed)
    if isinstance(seed, (np.random.RandomState, np.random.Generator)):
        return seed
    raise ValueError(f'{seed!r} cannot seed a numpy.random.RandomState')


def _draws(rngs, dithers, crs, index_rows, N, P, first, fill, cross):
    '''The draws of one generation of several searches in scipy's order, in
    one native call on the generators' own bit generators (lmb_de_draws_many:
    numpy's algorithms restated, the same draws in the same order, search
    after search).  Per search s: the dithered scale rng.uniform(*dither)
    (returned in scale[s]; NaN without dither), N times
    rng.shuffle(index_rows[s]) keeping its first three entries in first[s]
    (N, 3), fill[s] (N,) = the crossover's forced parameters, cross[s]
    (N, P) = rng.uniform(size=(N, P)) < crs[s].'''
    S = len(rngs)
    bgs = [r.bit_generator if isinstance(r, np.random.Generator)
           else r._bit_generator for r in rngs]
    ptrs = np.array([bg.ctypes.bit_generator.value for bg in bgs],
                    dtype=np.uintp)
    masked = np.array([not isinstance(r, np.random.Generator) for r in rngs],
                      dtype=np.int32)
    has = np.array([d is not None for d in dithers], dtype=np.int32)
    lo = np.array([d[0] if d is not None else 0. for d in dithers], dtype=float)
    hi = np.array([d[1] if d is not None else 0. for d in dithers], dtype=float)
    cr = np.ascontiguousarray(crs, dtype=float)
    rows = np.array([r.ctypes.data for r in index_rows], dtype=np.uintp)
    scale = np.empty(S)
    locks = {id(bg): bg.lock for bg in bgs}
    held = []
    try:
        for k in sorted(locks):
            locks[k].acquire()
            held.append(locks[k])
        st = _native.load().lmb_de_draws_many(
            S, ptrs.ctypes.data, masked.ctypes.data, has.ctypes.data,
            lo.ctypes.data, hi.ctypes.data, scale.ctypes.data,
            rows.ctypes.data, N, first.shape[-1], first.ctypes.data, P,
            cr.ctypes.data, fill.ctypes.data, cross.ctypes.data)
    finally:
        for lock in held:
            lock.release()
    _native.check(st, 'lmb_de_draws_many')
    scale[has == 0] = np.nan
    return scale


class Populations:
    '''Searches with the same population shape (N candidates, P
    parameters), stepped together: population (S, N, P) in [0, 1],
    energies (S, N).  Each search draws from its own generator in scipy's
    order; the arithmetic runs once for all of them (elementwise the same
    operations, so every value is the one a lone search computes).

    request(live) gives {search: parameters (N, P)} for the searches in
    ``live``; receive({search: energies (N,)}) advances them.  ``done[s]``
    is set, with ``results[s]``, when search s has converged or reached
    maxiter.'''

    def __init__(self, problems):
        S = len(problems)
        self.rngs, dither, scale, cr, tol, atol, maxiter = [], [], [], [], [], [], []
        mids, spans, pops = [], [], []
        for pr in problems:
            s = dict(_DEFAULTS)
            s.update(pr['settings'] or {})
            limits = np.array(pr['bounds'], dtype=float).T
            if limits.shape[0] != 2 or not np.all(np.isfinite(limits)):
                raise ValueError('bounds should be a sequence containing '
                                 'finite real valued (min, max) pairs for '
                                 'each value in x')
            mutation = s['mutation']
            d = None
            if hasattr(mutation, '__iter__') and len(mutation) > 1:
                d = sorted([mutation[0], mutation[1]])
            dither.append(d)
            scale.append(np.nan if d is not None else float(mutation))
            cr.append(s['recombination'])
            tol.append(s['tol'])
            atol.append(s['atol'])
            maxiter.append(1000 if s['maxiter'] is None else int(s['maxiter']))
            mids.append(0.5 * (limits[0] + limits[1]))
            spans.append(np.fabs(limits[0] - limits[1]))
            nparam = limits.shape[1]
            fixed = np.count_nonzero(limits[0] == limits[1])
            N = max(5, pr['popsize'] * max(1, nparam - fixed))
            rng = _generator(pr['seed'])
            self.rngs.append(rng)
            # latin hypercube: one draw per cell, one permutation per column
            seg = 1.0 / N
            samples = (seg * rng.uniform(size=(N, nparam)) +
                       np.linspace(0., 1., N, endpoint=False)[:, None])
            pop = np.zeros_like(samples)
            for j in range(nparam):
                order = rng.permutation(range(N))
                pop[:, j] = samples[order, j]
            pops.append(pop)
        self.S, self.N, self.P = S, pops[0].shape[0], pops[0].shape[1]
        self.dither = dither
        self.scale = np.array(scale, dtype=float)
        self.cr = np.array(cr, dtype=float)
        self.tol = np.array(tol, dtype=float)
        self.atol = np.array(atol, dtype=float)
        self.maxiter = np.array(maxiter)
        self.mid = np.array(mids)[:, None, :]
        self.span = np.array(spans)[:, None, :]
        self.pop = np.array(pops)
        self.energies = np.full((S, self.N), np.inf)
        self.trial = np.zeros_like(self.pop)
        self.index = np.tile(np.arange(self.N, dtype=np.int64), (S, 1))
        self.trialed = np.zeros(S, dtype=bool)   # last request was a trial
        self.nfev = np.zeros(S, dtype=int)
        self.nit = np.zeros(S, dtype=int)
        self.done = np.zeros(S, dtype=bool)
        self.results = [None] * S

    def parameters(self, s, unit):
        return self.mid[s, 0] + (unit - 0.5) * self.span[s, 0]

    def request(self, live):
        live = np.asarray(live)
        inf_all = np.all(np.isinf(self.energies[live]), axis=1)
        out = {}
        for s in live[inf_all]:               # (re)evaluate the population
            self.trialed[s] = False
            out[s] = self.parameters(s, self.pop[s])
        T = live[~inf_all]
        if not len(T):
            return out
        N, P = self.N, self.P
        first = np.empty((len(T), N, 3), dtype=self.index[0].dtype)
        fill = np.empty((len(T), N), dtype='int64')
        cross = np.empty((len(T), N, P), dtype=bool)
        # dithered scale; mutation, best1: for each candidate the first two
        # of a fresh shuffle of the kept permutation other than the
        # candidate; binomial crossover's forced parameter and draws
        scale = _draws([self.rngs[s] for s in T],
                       [self.dither[s] for s in T], self.cr[T],
                       [self.index[s] for s in T], N, P, first, fill, cross)
        dithered = ~np.isnan(scale)
        self.scale[T[dithered]] = scale[dithered]
        c = np.arange(N)
        f0, f1, f2 = first[..., 0], first[..., 1], first[..., 2]
        r0 = np.where(f0 == c, f1, f0)
        r1 = np.where((f0 == c) | (f1 == c), f2, f1)
        pop = self.pop[T]
        b0 = np.take_along_axis(pop, r0[..., None], axis=1)
        b1 = np.take_along_axis(pop, r1[..., None], axis=1)
        bprime = pop[:, :1, :] + self.scale[T][:, None, None] * (b0 - b1)
        cross[np.arange(len(T))[:, None], c[None, :], fill] = True
        trial = np.where(cross, bprime, pop)
        outside = (trial > 1) | (trial < 0)
        for i, s in enumerate(T):
            n = np.count_nonzero(outside[i])
            if n:
                trial[i][outside[i]] = self.rngs[s].uniform(size=n)
        self.trial[T] = trial
        self.trialed[T] = True
        params = self.mid[T] + (trial - 0.5) * self.span[T]
        for i, s in enumerate(T):
            out[s] = params[i]
        return out

    def receive(self, values):
        keys = np.array(sorted(values))
        E = np.array([np.asarray(values[s], dtype=float).reshape(-1)
                      for s in keys])
        self.nfev[keys] += 1
        fresh = ~self.trialed[keys]
        R = keys[fresh]                      # population (re)evaluated
        if len(R):
            self.energies[R] = E[fresh]
            self._promote(R)
        T = keys[~fresh]
        if not len(T):
            return
        Et = E[~fresh]
        keep = Et <= self.energies[T]
        self.pop[T] = np.where(keep[..., None], self.trial[T], self.pop[T])
        self.energies[T] = np.where(keep, Et, self.energies[T])
        self._promote(T)
        self.trialed[T] = False
        self.nit[T] += 1
        e = self.energies[T]
        conv = ~np.any(np.isinf(e), axis=1) & (
            np.std(e, axis=1) <= self.atol[T] + self.tol[T] * np.abs(
                np.mean(e, axis=1)))
        for i, s in enumerate(T):
            if conv[i]:
                self._finish(s, _SUCCESS, True)
            elif self.nit[s] >= self.maxiter[s]:
                self._finish(s, _MAXITER, False)

    def _promote(self, rows):
        best = np.argmin(self.energies[rows], axis=1)
        e0 = self.energies[rows, 0].copy()
        self.energies[rows, 0] = self.energies[rows, best]
        self.energies[rows, best] = e0
        p0 = self.pop[rows, 0, :].copy()
        self.pop[rows, 0, :] = self.pop[rows, best, :]
        self.pop[rows, best, :] = p0

    def _finish(self, s, message, success):
        self.done[s] = True
        self.results[s] = OptimizeResult(
            x=self.parameters(s, self.pop[s, 0]), fun=self.energies[s, 0],
            nfev=int(self.nfev[s]), nit=int(self.nit[s]), message=message,
            success=success, population=self.parameters(s, self.pop[s]),
            population_energies=self.energies[s].copy())


def _shape(problem):
    limits = np.array(problem['bounds'], dtype=float).T
    nparam = limits.shape[1] if limits.ndim == 2 else 0
    fixed = np.count_nonzero(limits[0] == limits[1]) if nparam else 0
    return max(5, problem['popsize'] * max(1, nparam - fixed)), nparam


def run_populations(problems, evaluate):
    '''Every problem (dict with bounds, popsize, seed, settings) searched
    with the others: each round, the parameters every unfinished search
    needs go to ``evaluate({index: x})`` at once (x as a vectorized scipy
    objective receives it, (P, N)); returns the OptimizeResults in order.
    Searches of the same population shape share arrays (Populations).'''
    groups = {}
    for i, p in enumerate(problems):
        groups.setdefault(_shape(p), []).append(i)
    parts = [(idx, Populations([problems[i] for i in idx]))
             for idx in groups.values()]
    while True:
        batch, owners = {}, []
        for idx, g in parts:
            live = np.flatnonzero(~g.done)
            if len(live):
                req = g.request(live)
                for s, x in req.items():
                    batch[idx[s]] = x.T
                owners.append((idx, g, list(req)))
        if not batch:
            break
        values = evaluate(batch)
        for idx, g, members in owners:
            g.receive({s: values[idx[s]] for s in members})
    results = [None] * len(problems)
    for idx, g in parts:
        for s, i in enumerate(idx):
            results[i] = g.results[s]
    return results
