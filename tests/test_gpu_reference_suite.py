'''GPU: the reference's own hot-path tests and Optimizer, run on this
package's model classes.

The reference installed into baseline/_ref (its package, plus its tests/
directory beside it) provides:

* its test modules tests/test_lorenzmie.py, test_sphere.py,
  test_instrument.py and test_optimizer.py, imported from that copy with
  their model classes re-pointed at pylorenzmie_b200's LorenzMie, Sphere
  and Instrument.  The reference's own Optimizer stays in place, so the
  optimizer tests drive our model through the reference's fitting code.
  The jax-only class TestOptimizerAnalyticalJac runs too, with our model in
  the jaxLorenzMie slot: the reference Optimizer then takes our jac()
  through _analytical_jac (analysis/Optimizer.py:218-220, 251-255);
* a fit by the reference's Optimizer with our model, compared with the
  reference's own fit of the same hologram (tests/golden/fit.npz).

Two reference tests state choices this package makes differently, and
are skipped with the reason: the model's method string ('b200 numpy',
which the reference Optimizer accepts by its substring rule,
analysis/Optimizer.py:64-65) and the analytic Jacobian's coverage of k_p
(this jac() has a k_p column; the reference's JAX one does not,
theory/jaxLorenzMie.py:321).

Install the reference there with (the checkout at REF):
    python -m pip install --no-index --no-build-isolation --no-deps \\
        --target baseline/_ref REF
    cp -r REF/tests baseline/_ref/tests
Without it these tests are skipped.
'''
import importlib.util
import sys
import types
import unittest
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent
REF = ROOT / 'baseline' / '_ref'
REF_TESTS = REF / 'tests'
MODULES = ('test_lorenzmie', 'test_sphere', 'test_instrument',
           'test_optimizer')
DIFFERENT = {
    ('test_lorenzmie', 'TestLorenzMie', 'test_method'):
        "method is 'b200 numpy', accepted by the reference Optimizer's "
        'substring rule',
    ('test_optimizer', 'TestOptimizerAnalyticalJac',
     'test_analytical_jac_skipped_for_uncovered_variable'):
        'this jac() covers k_p, so the analytic Jacobian is used with k_p '
        'free',
}


def _available():
    return (REF / 'pylorenzmie').is_dir() and all(
        (REF_TESTS / f'{m}.py').exists() for m in MODULES)


def _import_reference():
    if str(REF) not in sys.path:
        sys.path.insert(0, str(REF))
    if 'trackpy' not in sys.modules:   # imported by analysis/Localizer.py
        sys.modules['trackpy'] = types.ModuleType('trackpy')
    import pylorenzmie  # noqa: F401


def _load(name):
    '''The reference test module, re-pointed at this package's classes.'''
    _import_reference()
    import pylorenzmie_b200 as b
    spec = importlib.util.spec_from_file_location(
        f'reference_{name}', REF_TESTS / f'{name}.py')
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    for attr, cls in (('LorenzMie', b.LorenzMie), ('Sphere', b.Sphere),
                      ('Instrument', b.Instrument),
                      ('jaxLorenzMie', b.LorenzMie)):
        if hasattr(mod, attr) or attr == 'jaxLorenzMie':
            setattr(mod, attr, cls)
    for obj in vars(mod).values():
        if isinstance(obj, type) and issubclass(obj, unittest.TestCase):
            obj.__unittest_skip__ = False
    return mod


def _cases():
    if not _available():
        return [pytest.param(None, None, None, marks=pytest.mark.skip(
            reason='reference not installed in baseline/_ref'))]
    out = []
    for name in MODULES:
        src = (REF_TESTS / f'{name}.py').read_text()
        for line in src.splitlines():
            if line.startswith('class ') and 'TestCase' in line:
                cls = line.split()[1].split('(')[0]
                body = src.split(line, 1)[1].split('\nclass ', 1)[0]
                for bl in body.splitlines():
                    s = bl.strip()
                    if s.startswith('def test'):
                        meth = s[4:].split('(')[0]
                        marks = []
                        why = DIFFERENT.get((name, cls, meth))
                        if why:
                            marks = [pytest.mark.skip(reason=why)]
                        out.append(pytest.param(name, cls, meth, marks=marks,
                                                id=f'{name}.{cls}.{meth}'))
    return out


_MODS = {}


@pytest.mark.parametrize('name,cls,meth', _cases())
def test_reference_test_on_b200_classes(name, cls, meth):
    if name not in _MODS:
        _MODS[name] = _load(name)
    case = getattr(_MODS[name], cls)(meth)
    result = unittest.TestResult()
    case.run(result)
    problems = result.failures + result.errors
    assert not problems, problems[0][1]
    assert result.testsRun == 1 and not result.skipped, result.skipped


@pytest.mark.skipif(not _available(), reason='reference not installed')
def test_reference_optimizer_fits_with_b200_model(golden_fit):
    '''The reference's Optimizer with our model (analytic Jacobian through
    _analytical_jac) on the golden hologram: the fit the reference made with
    its own model and forward differences, within the fit targets.'''
    _import_reference()
    from pylorenzmie.analysis.Optimizer import Optimizer as RefOptimizer
    from pylorenzmie.analysis.Hologram import Hologram as RefHologram
    import pylorenzmie_b200 as b
    data = golden_fit['data']
    shape = tuple(int(v) for v in golden_fit['shape'])
    start = golden_fit['start']
    model = b.LorenzMie(coordinates=b.LorenzMie.meshgrid(shape))
    model.instrument.wavelength = 0.447
    model.instrument.magnification = 0.048
    model.instrument.n_m = 1.340
    model.particle.r_p = list(start[:3])
    model.particle.a_p, model.particle.n_p = start[3], start[4]
    opt = RefOptimizer(model=model)
    calls = []
    jac = opt._analytical_jac
    opt._analytical_jac = lambda v: (calls.append(1), jac(v))[1]
    result = opt.optimize(RefHologram(data.reshape(shape)))
    assert calls, 'the reference Optimizer did not use our jac()'
    ref = dict(zip(golden_fit['keys'], golden_fit['values']))
    assert bool(result['success'])
    tol = {'x_p': 0.02, 'y_p': 0.02, 'z_p': 0.02, 'a_p': 1e-3, 'n_p': 1e-4}
    for k, t in tol.items():
        assert abs(result[k] - ref[k]) <= t, (k, result[k], ref[k])
    assert abs(result['redchi'] / ref['redchi'] - 1) < 1e-3
