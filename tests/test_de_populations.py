'''The thread-free form of scipy's differential evolution (run_populations)
against scipy.optimize.differential_evolution itself: for every setting the
estimators use, each search returns exactly what scipy returns for it
(solution, energies, whole final population, nit, nfev, message), with
int, RandomState, Generator and global-generator seeds, scalar and
dithered mutation, exits at maxiter, fixed bounds, NaN energies and the
re-evaluation of an all-infinite first population.'''
import numpy as np
import pytest
from scipy.optimize import differential_evolution

from pylorenzmie_b200.analysis._de import Populations, run_populations, supported
from pylorenzmie_b200.analysis._population import de_settings


def _objective(c, w, nan_band=None, inf_calls=0):
    calls = [0]

    def f(x):
        calls[0] += 1
        X = np.asarray(x, dtype=float).reshape(len(c), -1)
        v = np.sum(((X - np.asarray(c)[:, None]) / np.asarray(w)[:, None])
                   ** 2, axis=0)
        v = v + np.sin(3. * X[0]) ** 2            # a few local minima
        if nan_band is not None:
            v[(X[0] > nan_band[0]) & (X[0] < nan_band[1])] = np.nan
        if calls[0] <= inf_calls:
            v[:] = np.inf
        return v
    return f


def _cases():
    base = {'tol': 0.01, 'polish': False, 'updating': 'deferred',
            'workers': -1}
    return [
        dict(bounds=[(10., 600.), (0.25, 10.), (1., 3.)], popsize=10,
             seed=3, settings=dict(base),
             f=(_objective, ([200., 1., 1.5], [100., 0.3, 0.1]))),
        dict(bounds=[(-2., 2.), (-2., 2.)], popsize=7,
             seed=np.random.RandomState(11),
             settings=dict(base, tol=1e-4, mutation=0.8, recombination=0.5),
             f=(_objective, ([0.3, -0.2], [1., 1.]))),
        dict(bounds=[(-2., 2.), (0.5, 0.5), (0., 1.)], popsize=6,
             seed=np.random.default_rng(5),
             settings=dict(base, maxiter=7),
             f=(_objective, ([0.1, 0.5, 0.4], [1., 1., 0.3]))),
        dict(bounds=[(-3., 3.)] * 4, popsize=5, seed=19,
             settings=dict(base, tol=0., atol=1e-3, maxiter=40,
                           mutation=(0.2, 1.5)),
             f=(_objective, ([0.5, 0.1, -0.3, 1.], [1., 2., 1., 0.5]),
                {'nan_band': (-0.5, 0.2)})),
        dict(bounds=[(0., 5.), (0., 5.)], popsize=8, seed=23,
             settings=dict(base),
             f=(_objective, ([2., 3.], [1., 1.]), {'inf_calls': 1})),
    ]


def _fresh_seed(seed, k):
    # an equal, independent generator for each of the two runs
    if isinstance(seed, np.random.RandomState):
        return np.random.RandomState(11)
    if isinstance(seed, np.random.Generator):
        return np.random.default_rng(5)
    return seed


def _make(case):
    fn, args, *kw = case['f']
    return fn(*args, **(kw[0] if kw else {}))


def _scipy(case, k):
    f = _make(case)
    with np.errstate(invalid='ignore'):
        return differential_evolution(f, case['bounds'],
                                      popsize=case['popsize'],
                                      seed=_fresh_seed(case['seed'], k),
                                      **de_settings(case['settings']))


def _assert_same(r, ref):
    np.testing.assert_array_equal(r.x, ref.x)
    np.testing.assert_array_equal(r.population, ref.population)
    np.testing.assert_array_equal(r.population_energies,
                                  ref.population_energies)
    assert (r.fun == ref.fun) or (np.isnan(r.fun) and np.isnan(ref.fun))
    assert (r.nit, r.nfev, r.message, r.success) == \
        (ref.nit, ref.nfev, ref.message, ref.success)


def test_each_search_matches_scipy_alone():
    cases = _cases()
    for k, case in enumerate(cases):
        assert supported(case['settings'])
        f = _make(case)
        pr = dict(case, seed=_fresh_seed(case['seed'], k))
        with np.errstate(invalid='ignore'):
            r = run_populations([pr], lambda b: {0: f(b[0])})[0]
        _assert_same(r, _scipy(case, k))


def test_searches_together_match_scipy():
    '''All cases stepped together (each evaluation sees every unfinished
    search); seeded searches are unaffected by their companions.'''
    cases = _cases()
    fs = [_make(c) for c in cases]
    problems = [dict(c, seed=_fresh_seed(c['seed'], k))
                for k, c in enumerate(cases)]
    rounds = []

    def evaluate(batch):
        rounds.append(sorted(batch))
        return {i: fs[i](x) for i, x in batch.items()}
    with np.errstate(invalid='ignore'):
        got = run_populations(problems, evaluate)
    for k, (case, r) in enumerate(zip(cases, got)):
        _assert_same(r, _scipy(case, k))
    assert rounds[0] == list(range(len(cases)))
    assert len(rounds) == max(r.nfev for r in got)


def test_global_generator_search_matches_scipy():
    case = _cases()[0]
    f = _make(case)
    np.random.seed(31)
    r = run_populations([dict(case, seed=None)], lambda b: {0: f(b[0])})[0]
    np.random.seed(31)
    ref = differential_evolution(_make(case), case['bounds'],
                                 popsize=case['popsize'], seed=None,
                                 **de_settings(case['settings']))
    _assert_same(r, ref)


@pytest.mark.parametrize('extra', [{'polish': True}, {'strategy': 'rand1bin'},
                                   {'init': 'sobol'}, {'maxfun': 100},
                                   {'x0': [1., 1.]}, {'callback': print},
                                   {'mutation': (0.5, 2.5)}, {'maxiter': 0},
                                   {'unknown': 1}])
def test_other_settings_go_to_scipy(extra):
    s = {'tol': 0.01, 'polish': False, 'updating': 'deferred'}
    assert supported(s)
    assert not supported(dict(s, **extra))


def test_bad_bounds_raise():
    with pytest.raises(ValueError):
        Populations([dict(bounds=[(0., np.inf)], popsize=5, seed=1,
                          settings={})])


def test_one_shape_group_matches_scipy():
    '''Twelve searches of one population shape share arrays: different
    objectives, generators, tolerances, mutation settings and maxiter
    exits, a NaN band, and a search whose first population is all
    infinite; each still ends where scipy ends alone.'''
    base = {'tol': 0.01, 'polish': False, 'updating': 'deferred',
            'workers': -1}
    rng = np.random.default_rng(17)
    cases = []
    for i in range(12):
        c = list(rng.uniform(-1., 1., 3))
        kw = {}
        if i == 4:
            kw['nan_band'] = (-0.3, 0.1)
        if i == 7:
            kw['inf_calls'] = 1
        settings = dict(base, tol=[0.01, 1e-3, 0.05][i % 3])
        if i % 4 == 1:
            settings['mutation'] = 0.7
        if i % 5 == 2:
            settings['maxiter'] = 6
        if i % 6 == 3:
            settings['recombination'] = 0.4
        seed = (100 + i if i % 3 == 0 else
                np.random.RandomState(200 + i) if i % 3 == 1 else
                np.random.default_rng(300 + i))
        cases.append((dict(bounds=[(-2., 2.)] * 3, popsize=10,
                           settings=settings), c, kw, i))

    def fresh(i):
        return (100 + i if i % 3 == 0 else
                np.random.RandomState(200 + i) if i % 3 == 1 else
                np.random.default_rng(300 + i))
    fs = [_objective(c, [1., 0.5, 0.3], **kw) for _, c, kw, _ in cases]
    problems = [dict(p, seed=fresh(i)) for p, _, _, i in cases]
    with np.errstate(invalid='ignore'):
        got = run_populations(problems, lambda b: {k: fs[k](x)
                                                   for k, x in b.items()})
    for (p, c, kw, i), r in zip(cases, got):
        f = _objective(c, [1., 0.5, 0.3], **kw)
        with np.errstate(invalid='ignore'):
            ref = differential_evolution(f, p['bounds'], popsize=10,
                                         seed=fresh(i),
                                         **de_settings(p['settings']))
        _assert_same(r, ref)
    assert len({r.nit for r in got}) > 3      # they finished apart


def _pair(kind, seed):
    if kind == 'RandomState':
        return np.random.RandomState(seed), np.random.RandomState(seed)
    return np.random.default_rng(seed), np.random.default_rng(seed)


def _bitgen(rng):
    return (rng.bit_generator if isinstance(rng, np.random.Generator)
            else rng._bit_generator)


@pytest.mark.parametrize('kind', ['RandomState', 'Generator'])
def test_native_shuffles_are_numpys(kind):
    '''lmb_de_shuffles against numpy's shuffle: the same permutations and
    the same state after, from any point of the stream (an odd number of
    32-bit draws consumed too), for sizes 0 to past 2**16.'''
    from pylorenzmie_b200 import _native
    lib = _native.load()
    for seed in range(12):
        for n in (0, 1, 2, 3, 30, 33, 70000):
            a, b = _pair(kind, seed)
            for r in (a, b):
                r.uniform(size=3)
                r.randint(7) if kind == 'RandomState' else r.integers(7)
            count = 3 if n > 1000 else 20
            keep = min(3, n)
            ia, ib = np.arange(n), np.arange(n, dtype=np.int64)
            ref = np.empty((count, keep), dtype=np.int64)
            for c in range(count):
                a.shuffle(ia)
                ref[c] = ia[:keep]
            out = np.empty((count, keep), dtype=np.int64)
            bg = _bitgen(b)
            with bg.lock:
                assert lib.lmb_de_shuffles(bg.ctypes.bit_generator,
                                           ib.ctypes.data, n, count, keep,
                                           out.ctypes.data) == 0
            np.testing.assert_array_equal(out, ref)
            np.testing.assert_array_equal(ib, ia)
            assert a.uniform() == b.uniform()


def _numpy_draws(rng, dither, index, N, P, cr):
    '''One search's generation of draws by numpy's own calls, scipy's
    order.'''
    scale = rng.uniform(*dither) if dither else np.nan
    first = np.empty((N, 3), dtype=np.int64)
    for c in range(N):
        rng.shuffle(index)
        first[c] = index[:3]
    fill = (rng.integers(P, size=N, dtype='int64')
            if isinstance(rng, np.random.Generator) else
            rng.randint(P, size=N, dtype='int64'))
    return scale, first, fill, rng.uniform(size=(N, P)) < cr


def test_native_generation_draws_are_numpys():
    '''_draws (lmb_de_draws_many: a generation of several searches' draws
    in one native call) against the numpy calls scipy makes, search after
    search: the dithered scale, the N shuffles, the crossover's forced
    parameters (RandomState.randint / Generator.integers) and the crossover
    uniforms; identical values and the same generator states after, with
    RandomState and Generator searches mixed and two searches sharing one
    generator.'''
    from pylorenzmie_b200.analysis._de import _draws
    for seed in range(8):
        for N, P in ((5, 1), (30, 3), (31, 5), (60, 6)):
            def make():
                shared = np.random.RandomState(seed + 100)
                rngs = [np.random.RandomState(seed),
                        np.random.default_rng(seed), shared,
                        np.random.default_rng(seed + 1), shared]
                for r in rngs[:4]:
                    r.uniform(size=seed % 3)
                return rngs
            ra, rb = make(), make()
            dithers = [None, (0.5, 1.0), (0.4, 0.9), None, (0.5, 1.0)]
            crs = np.array([0.7, 0.9, 0.5, 0.7, 0.3])
            S = len(ra)
            ia = np.tile(np.arange(N, dtype=np.int64), (S, 1))
            ib = ia.copy()
            ref = [_numpy_draws(ra[s], dithers[s], ia[s], N, P, crs[s])
                   for s in range(S)]
            first = np.empty((S, N, 3), dtype=np.int64)
            fill = np.empty((S, N), dtype=np.int64)
            cross = np.empty((S, N, P), dtype=bool)
            scale = _draws(rb, dithers, crs, [ib[s] for s in range(S)], N, P,
                           first, fill, cross)
            for s in range(S):
                np.testing.assert_array_equal(scale[s], ref[s][0])
                np.testing.assert_array_equal(first[s], ref[s][1])
                np.testing.assert_array_equal(fill[s], ref[s][2])
                np.testing.assert_array_equal(cross[s], ref[s][3])
            np.testing.assert_array_equal(ib, ia)
            for a, b in zip(ra, rb):
                assert a.uniform() == b.uniform()
