'''Host logic of side-by-side differential-evolution searches (lockstep_de):
every search ends exactly where scipy's differential_evolution ends alone
with the same settings, however many worker threads share the generations;
an error of one search or of the evaluation reaches the caller.  The
objective here is numpy (no GPU); on the GPU it is one lmb_chi2_crops
launch per generation (tests/test_gpu_estimate.py).'''
import numpy as np
import pytest
from scipy.optimize import differential_evolution

from pylorenzmie_b200.analysis._population import de_settings, lockstep_de


def _shifted_rosen(c):
    def f(x):
        x = np.asarray(x, dtype=float)
        X = x.reshape(len(c), -1) - np.asarray(c)[:, None]
        v = np.sum(100. * (X[1:] - X[:-1] ** 2) ** 2 + (1. - X[:-1]) ** 2,
                   axis=0)
        return float(v[0]) if x.ndim == 1 else v
    return f


def _problems(n):
    rng = np.random.default_rng(5)
    out = []
    for i in range(n):
        nvar = 2 + i % 3
        c = rng.uniform(-0.5, 0.5, nvar)
        out.append(dict(bounds=[(-2., 2.)] * nvar, popsize=5 + i % 4,
                        seed=100 + i,
                        settings={'tol': 0.01 * (1 + i % 2), 'polish': False,
                                  'updating': 'deferred', 'workers': -1},
                        f=_shifted_rosen(c)))
    return out


def _alone(pr):
    return differential_evolution(pr['f'], pr['bounds'], popsize=pr['popsize'],
                                  seed=pr['seed'],
                                  **de_settings(pr['settings']))


@pytest.mark.parametrize('workers', [1, 3, 64])
def test_lockstep_matches_each_search_alone(workers):
    problems = _problems(9)
    calls = []

    def evaluate(batch):
        calls.append(len(batch))
        return {i: problems[i]['f'](x) for i, x in batch.items()}

    got = lockstep_de(problems, evaluate, workers=workers)
    for pr, r in zip(problems, got):
        ref = _alone(pr)
        np.testing.assert_array_equal(r.x, ref.x)
        assert r.fun == ref.fun and r.nit == ref.nit and r.nfev == ref.nfev
    # searches shared generations: fewer evaluations than objective calls
    assert max(calls) == min(workers, len(problems))
    assert sum(calls) == sum(r.nit + 1 for r in got)


def test_lockstep_empty():
    assert lockstep_de([], lambda b: {}) == []


def test_lockstep_evaluation_error_reaches_caller():
    problems = _problems(4)
    n = [0]

    def evaluate(batch):
        n[0] += 1
        if n[0] == 3:
            raise RuntimeError('evaluation failed')
        return {i: problems[i]['f'](x) for i, x in batch.items()}

    with pytest.raises(RuntimeError, match='evaluation failed'):
        lockstep_de(problems, evaluate, workers=4)


def test_lockstep_search_error_reaches_caller():
    problems = _problems(4)
    problems[2]['settings'] = dict(problems[2]['settings'], mutation=3.)

    def evaluate(batch):
        return {i: problems[i]['f'](x) for i, x in batch.items()}

    with pytest.raises(ValueError, match='mutation'):
        lockstep_de(problems, evaluate, workers=2)
