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
import numbers

import numpy as np
from scipy.optimize import OptimizeResult

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


def _integers(rng, high, size):
    '''Integers in [0, high), as scipy's rng_integers.'''
    if isinstance(rng, np.random.Generator):
        return rng.integers(high, size=size, dtype='int64')
    return rng.randint(high, size=size, dtype='int64')


class Population:
    '''One search's state: population (N, P) in [0, 1], energies (N,).

    request() gives the parameters (N, P) the search needs evaluated next;
    receive(energies) takes their values and advances it.  ``done`` is set
    with ``result`` when it has converged or reached maxiter.'''

    def __init__(self, bounds, popsize=15, seed=None, settings=None):
        s = dict(_DEFAULTS)
        s.update(settings or {})
        limits = np.array(bounds, dtype=float).T
        if limits.shape[0] != 2 or not np.all(np.isfinite(limits)):
            raise ValueError('bounds should be a sequence containing finite '
                             'real valued (min, max) pairs for each value '
                             'in x')
        self.tol, self.atol = s['tol'], s['atol']
        self.maxiter = 1000 if s['maxiter'] is None else int(s['maxiter'])
        mutation = s['mutation']
        self.scale = mutation
        self.dither = None
        if hasattr(mutation, '__iter__') and len(mutation) > 1:
            self.dither = sorted([mutation[0], mutation[1]])
        self.cr = s['recombination']
        self.limits = limits
        self._mid = 0.5 * (limits[0] + limits[1])
        self._span = np.fabs(limits[0] - limits[1])
        self.nparam = limits.shape[1]
        self.rng = _generator(seed)
        fixed = np.count_nonzero(limits[0] == limits[1])
        self.N = max(5, popsize * max(1, self.nparam - fixed))
        # latin hypercube: one draw per cell, one permutation per column
        rng = self.rng
        seg = 1.0 / self.N
        samples = (seg * rng.uniform(size=(self.N, self.nparam)) +
                   np.linspace(0., 1., self.N, endpoint=False)[:, None])
        self.population = np.zeros_like(samples)
        for j in range(self.nparam):
            order = rng.permutation(range(self.N))
            self.population[:, j] = samples[order, j]
        self.energies = np.full(self.N, np.inf)
        self._index = np.arange(self.N)
        self._first = np.empty((self.N, 3), dtype=self._index.dtype)
        self._trial = None
        self.nfev = 0
        self.nit = 0
        self.done = False
        self.result = None

    def parameters(self, unit):
        return self._mid + (unit - 0.5) * self._span

    def request(self):
        if np.all(np.isinf(self.energies)):
            self._trial = None           # (re)evaluate the population
            return self.parameters(self.population)
        rng = self.rng
        if self.dither is not None:
            self.scale = rng.uniform(self.dither[0], self.dither[1])
        # mutation, best1: for each candidate the first two of a fresh
        # shuffle of the kept permutation other than the candidate itself
        shuffle, index, first = rng.shuffle, self._index, self._first
        for c in range(self.N):
            shuffle(index)
            first[c] = index[:3]
        c = np.arange(self.N)
        f0, f1, f2 = first[:, 0], first[:, 1], first[:, 2]
        r0 = np.where(f0 == c, f1, f0)
        r1 = np.where((f0 == c) | (f1 == c), f2, f1)
        pop = self.population
        bprime = pop[0] + self.scale * (pop[r0] - pop[r1])
        fill = _integers(rng, self.nparam, self.N)
        cross = rng.uniform(size=(self.N, self.nparam)) < self.cr
        cross[c, fill] = True
        trial = np.where(cross, bprime, pop)
        out = (trial > 1) | (trial < 0)
        n = np.count_nonzero(out)
        if n:
            trial[out] = rng.uniform(size=n)
        self._trial = trial
        return self.parameters(trial)

    def receive(self, energies):
        energies = np.asarray(energies, dtype=float).reshape(-1)
        self.nfev += 1
        if self._trial is None:
            self.energies = energies.copy()
            self._promote()
            return
        keep = energies <= self.energies
        self.population = np.where(keep[:, None], self._trial,
                                   self.population)
        self.energies = np.where(keep, energies, self.energies)
        self._promote()
        self._trial = None
        self.nit += 1
        if self._converged():
            self._finish(_SUCCESS, True)
        elif self.nit >= self.maxiter:
            self._finish(_MAXITER, False)

    def _promote(self):
        best = int(np.argmin(self.energies))
        self.energies[[0, best]] = self.energies[[best, 0]]
        self.population[[0, best], :] = self.population[[best, 0], :]

    def _converged(self):
        e = self.energies
        if np.any(np.isinf(e)):
            return False
        return np.std(e) <= self.atol + self.tol * np.abs(np.mean(e))

    def _finish(self, message, success):
        self.done = True
        self.result = OptimizeResult(
            x=self.parameters(self.population[0]), fun=self.energies[0],
            nfev=self.nfev, nit=self.nit, message=message, success=success,
            population=self.parameters(self.population),
            population_energies=self.energies)


def run_populations(problems, evaluate):
    '''Every problem (dict with bounds, popsize, seed, settings) searched
    with the others: each round, the parameters every unfinished search
    needs go to ``evaluate({index: x})`` at once (x as a vectorized scipy
    objective receives it, (P, N)); returns the OptimizeResults in order.'''
    searches = [Population(p['bounds'], p['popsize'], p['seed'],
                           p['settings']) for p in problems]
    live = list(range(len(searches)))
    while live:
        batch = {i: searches[i].request().T for i in live}
        values = evaluate(batch)
        for i in live:
            searches[i].receive(values[i])
        live = [i for i in live if not searches[i].done]
    return [s.result for s in searches]
