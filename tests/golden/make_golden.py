'''Generate the golden fixtures of tests/golden/ by running the reference.

Run from the repository root on a machine that has the reference checkout,
naming it with ``--reference`` or the ``LM_REFERENCE`` environment variable:

    python tests/golden/make_golden.py --reference PATH [fixture ...]

(no fixture names: all of them).  The reference package is made importable
as ``pylorenzmie`` through a symlink in a temporary directory, with an empty
``trackpy`` stub (its analysis/__init__.py imports Localizer, which imports
trackpy).  The numpy FP64 model is imported explicitly from
``pylorenzmie.theory.LorenzMie`` because the package-level ``LorenzMie``
resolves to the fastmath numba backend (theory/__init__.py:33-38).

Outputs (small, committed):
  ab.npz        Sphere.mie_coefficients for a table of spheres
  layered.npz   sphere_coefficients: one layer (scalar input, as the
                reference accepts it) and 2- to 4-layer spheres (the
                reference's recurrences with its input handling repaired;
                see reference_layered below)
  holo.npz      LorenzMie.field/hologram for the reference tests' geometries
  fit.npz       a seeded 201x201 fit by the reference Optimizer
  estimate.npz  seeded DEEstimator and RadialEstimator searches (81x81 crop)
  variants.npz  AberratedLorenzMie and Dimer holograms
'''
import argparse
import os
import sys
import tempfile
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REFERENCE = None  # set by main()


def import_reference():
    tmp = Path(tempfile.mkdtemp(prefix='lmref_'))
    (tmp / 'pylorenzmie').symlink_to(REFERENCE)
    (tmp / 'trackpy.py').write_text('def locate(*a, **k):\n    raise '
                                    'RuntimeError("trackpy stub")\n')
    sys.path.insert(0, str(tmp))
    import pylorenzmie  # noqa: F401
    return tmp


# sphere table: (a_p, n_p, k_p, n_m, wavelength)
AB_CASES = [
    (0.75, 1.42, 0.0, 1.340, 0.447),      # the 201x201 single-sphere case
    (1.0, 1.40, 0.0, 1.34, 0.447),        # reference test_sphere setUp
    (0.4, 1.38, 0.0, 1.340, 0.447),
    (0.5, 1.45, 0.0, 1.340, 0.447),
    (1.5, 1.59, 0.0, 1.340, 0.447),
    (3.0, 1.70, 1e-3, 1.340, 0.447),      # frame-case upper corner
    (6.0, 2.00, 0.0, 1.340, 0.447),       # large-sphere upper corner
    (1.1, 1.40, 0.0, 1.34, 0.447),        # crop.png starting guess
    (0.8, 2.50, 0.05, 1.333, 0.532),      # absorbing, high index
    (0.05, 1.50, 0.0, 1.340, 0.447),      # Rayleigh-size sphere
]

WY_CASES = [(1., 10. + 0.j), (10., 10. + 0.j), (4210., 10. + 0.j),
            (5., 1.2), (100., 1.05 + 0.01j), (7.99, 1.5), (8.01, 1.5)]


def make_ab():
    from pylorenzmie.theory.Sphere import Sphere
    out = {}
    for i, (a_p, n_p, k_p, n_m, lam) in enumerate(AB_CASES):
        out[f'ab_{i}'] = Sphere.mie_coefficients(a_p, n_p, k_p, n_m, lam)
    out['cases'] = np.array(AB_CASES)
    out['wy_x'] = np.array([c[0] for c in WY_CASES])
    out['wy_m'] = np.array([c[1] for c in WY_CASES], dtype=complex)
    out['wy_n'] = np.array([Sphere.wiscombe_yang(x, m) for x, m in WY_CASES])
    out['np_x'] = np.array([1., 10., 55.5])
    out['np_n'] = np.array([Sphere.neves_pisignano(x) for x in out['np_x']])
    np.savez_compressed(HERE / 'ab.npz', **out)


# The reference's multilayer entry point (lib/obsolete/sphere_coefficients.py)
# cannot take more than one layer as written: it wraps its inputs in an
# extra dimension and counts layers by ndim (:85-87), checks the indices the
# same way (:89-90), and takes the builtin max of arrays in wiscombe_yang
# (:61).  These three replacements repair only that input handling, so that
# the recurrences of :126-215 run unchanged on 1-D radii and indices
# ordered from the core outwards.
LAYERED_INPUT_FIXES = [
    ('    a_p = np.array([a_p])\n    n_p = np.array([n_p])\n'
     '    nlayers = a_p.ndim\n',
     '    a_p = np.atleast_1d(np.asarray(a_p, dtype=float))\n'
     '    n_p = np.atleast_1d(np.asarray(n_p, dtype=complex))\n'
     '    nlayers = a_p.size\n'),
    ('    assert n_p.ndim == nlayers,', '    assert n_p.size == nlayers,'),
    ('    nstop = max(ns, xm, xm_1)',
     '    nstop = max(ns, np.max(xm), np.max(xm_1))'),
]


def reference_layered():
    '''The reference module's sphere_coefficients, executed from its own
    source file with LAYERED_INPUT_FIXES applied (each must match once).'''
    path = Path(REFERENCE) / 'lib' / 'obsolete' / 'sphere_coefficients.py'
    src = path.read_text()
    for old, new in LAYERED_INPUT_FIXES:
        if src.count(old) != 1:
            raise RuntimeError(f'reference source changed: {old!r}')
        src = src.replace(old, new)
    mod = types.ModuleType('reference_sphere_coefficients')
    mod.__file__ = str(path)
    exec(compile(src, str(path), 'exec'), mod.__dict__)
    return mod.sphere_coefficients


def layered_cases():
    '''Multilayer table: (radii core -> outer [um], indices core -> outer,
    n_m, wavelength).  The last four are seeded draws of the layered-stream
    workload (3 layers, fractions U(0.3, 0.9) nested, indices U(1.33,
    1.80), outer radius U(0.5, 2.5) um).'''
    cases = [([0.3, 0.75], [1.6, 1.45 + 0.002j], 1.34, 0.447),
             ([0.4, 0.8, 1.2], [1.8 + 0.01j, 1.33, 1.5], 1.34, 0.447),
             ([0.5, 1.25, 2.0], [1.4, 1.7, 1.55 + 0.001j], 1.34, 0.447),
             ([0.2, 0.35, 0.5, 0.9], [2.0, 1.4, 1.6, 1.38], 1.333, 0.532)]
    rng = np.random.default_rng(31)
    for _ in range(4):
        a = rng.uniform(0.5, 2.5)
        frac = np.sort(rng.uniform(0.3, 0.9, 2))
        idx = rng.uniform(1.33, 1.80, 3)
        cases.append((list(np.append(frac * a, a)), list(idx), 1.34, 0.447))
    return cases


def make_layered():
    from pylorenzmie.lib.obsolete.sphere_coefficients import \
        sphere_coefficients
    cases = [(0.75, 1.42, 1.340, 0.447), (1.2, 1.5 + 0.01j, 1.34, 0.447),
             (2.0, 1.6, 1.333, 0.532)]
    out = {'cases': np.array(cases, dtype=complex)}
    for i, (a, n, nm, lam) in enumerate(cases):
        out[f'ab_{i}'] = sphere_coefficients(a, n, nm, lam, resolution=None)
    repaired = reference_layered()
    multi = layered_cases()
    out['multi_count'] = np.array(len(multi))
    for i, (radii, idx, nm, lam) in enumerate(multi):
        out[f'multi_radii_{i}'] = np.array(radii, dtype=float)
        out[f'multi_indices_{i}'] = np.array(idx, dtype=complex)
        out[f'multi_medium_{i}'] = np.array([nm, lam])
        out[f'multi_ab_{i}'] = repaired(radii, idx, nm, lam, resolution=None)
    # the repaired entry point on one layer is the reference's own output
    # (to rounding: the index enters as complex instead of real)
    for i, (a, n, nm, lam) in enumerate(cases):
        ref = out[f'ab_{i}']
        got = repaired([a], [n], nm, lam, resolution=None)
        assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()
    np.savez_compressed(HERE / 'layered.npz', **out)


HOLO_CASES = [
    # name, shape, particles [(x,y,z,a,n,k)], cartesian, bohren
    ('torch64', (64, 64), [(32., 32., 150., 0.75, 1.45, 0.)], True, True),
    ('cupy128', (128, 128), [(64., 64., 100., 1.0, 1.4, 0.)], True, True),
    ('pair96', (96, 96), [(60., 70., 200., 0.5, 1.45, 0.),
                          (30., 10., 250., 1.0, 1.45, 0.)], True, True),
    ('absorb48', (48, 48), [(20.3, 25.7, 120., 0.9, 1.6, 0.01)], True, True),
    ('below40', (40, 40), [(20., 20., -130., 0.6, 1.5, 0.)], True, True),
    ('sph_nb32', (32, 32), [(16., 16., 100., 1.0, 1.4, 0.)], False, False),
    ('sph_b32', (32, 32), [(16., 16., 100., 1.0, 1.4, 0.)], False, True),
    ('cart_nb32', (32, 32), [(16., 16., 100., 1.0, 1.4, 0.)], True, False),
    ('big64', (64, 64), [(31.5, 30.25, 260., 3.0, 1.7, 0.001)], True, True),
]


def make_holo():
    from pylorenzmie.theory.LorenzMie import LorenzMie
    from pylorenzmie.theory.Sphere import Sphere
    from pylorenzmie.theory.Instrument import Instrument
    out = {}
    for name, shape, plist, cart, bohren in HOLO_CASES:
        inst = Instrument(wavelength=0.447, magnification=0.048, n_m=1.340)
        parts = []
        for (x, y, z, a, n, k) in plist:
            s = Sphere(a_p=a, n_p=n, k_p=k)
            s.r_p = [x, y, z]
            parts.append(s)
        coords = LorenzMie.meshgrid(shape)
        model = LorenzMie(coordinates=coords, particle=parts,
                          instrument=inst)
        fld = model.field(cartesian=cart, bohren=bohren).copy()
        holo = model.hologram(cartesian=cart, bohren=bohren)
        if fld.shape[1] <= 4096:
            out[f'{name}_field'] = fld
        out[f'{name}_holo'] = holo
        out[f'{name}_shape'] = np.array(shape)
        out[f'{name}_particles'] = np.array(plist)
        out[f'{name}_flags'] = np.array([cart, bohren])
    np.savez_compressed(HERE / 'holo.npz', **out)


def make_fit(seed=20240521):
    from pylorenzmie.theory.LorenzMie import LorenzMie
    from pylorenzmie.analysis.Optimizer import Optimizer
    from pylorenzmie.analysis.Hologram import Hologram
    rng = np.random.default_rng(seed)
    shape = (201, 201)
    truth = dict(x_p=100. + rng.uniform(-2, 2), y_p=100. + rng.uniform(-2, 2),
                 z_p=200., a_p=0.75, n_p=1.42, k_p=0.)
    model = LorenzMie(coordinates=LorenzMie.meshgrid(shape))
    model.instrument.wavelength = 0.447
    model.instrument.magnification = 0.048
    model.instrument.n_m = 1.340
    model.properties = truth
    clean = model.hologram().copy()
    data = clean + rng.normal(0., 0.05, size=clean.shape)
    start = dict(truth)
    start['a_p'] = truth['a_p'] * 1.05
    start['n_p'] = truth['n_p'] + 0.02
    start['z_p'] = truth['z_p'] + 10.
    model.properties = start
    opt = Optimizer(model=model)
    result = opt.optimize(Hologram(data.reshape(shape)))
    keys = list(result.index)
    np.savez_compressed(HERE / 'fit.npz', data=data, shape=np.array(shape),
                        truth=np.array([truth[k] for k in
                                        ('x_p', 'y_p', 'z_p', 'a_p', 'n_p',
                                         'k_p')]),
                        start=np.array([start[k] for k in
                                        ('x_p', 'y_p', 'z_p', 'a_p', 'n_p',
                                         'k_p')]),
                        keys=np.array(keys),
                        values=np.array([float(result[k]) for k in keys]),
                        nfev=np.array(opt._result.nfev),
                        status=np.array(opt._result.status),
                        seed=np.array(seed))


def make_estimate(seed=11):
    from pylorenzmie.theory.LorenzMie import LorenzMie
    from pylorenzmie.analysis.DEEstimator import DEEstimator
    from pylorenzmie.analysis.RadialEstimator import RadialEstimator
    from pylorenzmie.analysis.Hologram import Hologram
    rng = np.random.default_rng(seed)
    shape = (81, 81)
    truth = dict(x_p=40.3, y_p=39.7, z_p=150., a_p=0.75, n_p=1.42, k_p=0.)

    def model():
        m = LorenzMie(coordinates=LorenzMie.meshgrid(shape))
        m.instrument.wavelength = 0.447
        m.instrument.magnification = 0.048
        m.instrument.n_m = 1.340
        return m
    m = model()
    m.properties = truth
    data = (m.hologram() + rng.normal(0., 0.05, shape[0] * shape[1])
            ).reshape(shape)
    serial = {'tol': 0.01, 'polish': False, 'updating': 'deferred',
              'workers': 1}
    m = model()
    np.random.seed(7)  # the DE pixel subset (Mask draws from numpy's global RNG)
    de = DEEstimator(model=m, seed=3, settings=dict(serial)).estimate(
        Hologram(data))
    m = model()
    radial = RadialEstimator(model=m, seed=3, settings=dict(serial)).estimate(
        Hologram(data))
    keys = ('x_p', 'y_p', 'z_p', 'a_p', 'n_p', 'k_p')
    np.savez_compressed(HERE / 'estimate.npz', data=data,
                        truth=np.array([truth[k] for k in keys]),
                        de=np.array([float(de[k]) for k in keys]),
                        radial=np.array([float(radial[k]) for k in keys]),
                        mask_seed=np.array(7), de_seed=np.array(3),
                        seed=np.array(seed))


def make_variants():
    from pylorenzmie.theory.LorenzMie import LorenzMie
    from pylorenzmie.theory.Aberrated import Aberrated
    from pylorenzmie.theory.Sphere import Sphere
    from pylorenzmie.theory.Dimer import Dimer
    out = {}
    shape = (64, 72)
    coords = LorenzMie.meshgrid(shape)
    AbLM = Aberrated(LorenzMie)
    cases = [(0.9, (30.3, 35.2, 140., 0.8, 1.45, 0.)),
             (-2.5, (10.0, 60.0, 90., 1.2, 1.6, 0.002))]
    for i, (spherical, p) in enumerate(cases):
        s = Sphere(a_p=p[3], n_p=p[4], k_p=p[5])
        s.r_p = list(p[:3])
        m = AbLM(coordinates=coords, particle=s, spherical=spherical)
        m.instrument.wavelength = 0.447
        m.instrument.magnification = 0.048
        m.instrument.n_m = 1.340
        out[f'ab_holo_{i}'] = m.hologram()
        out[f'ab_case_{i}'] = np.array([spherical, *p])
    d = Dimer(magnification=0.048)
    d.a_p = 0.5
    d.n_p = 1.42
    d.r_p = [36., 30., 250.]
    d.theta = np.pi / 5.
    d.phi = np.pi / 3.
    m = LorenzMie(coordinates=coords, particle=d)
    m.instrument.wavelength = 0.447
    m.instrument.magnification = 0.048
    m.instrument.n_m = 1.340
    out['dimer_holo'] = m.hologram()
    out['dimer_case'] = np.array([36., 30., 250., 0.5, 1.42, 0., np.pi / 5.,
                                  np.pi / 3.])
    out['dimer_spheres'] = np.array([[*(q.r_p + q.r_0), q.a_p, q.n_p, q.k_p]
                                     for q in d.particles])
    out['shape'] = np.array(shape)
    np.savez_compressed(HERE / 'variants.npz', **out)


MAKERS = {'ab': lambda: make_ab(), 'layered': lambda: make_layered(),
          'holo': lambda: make_holo(), 'fit': lambda: make_fit(),
          'estimate': lambda: make_estimate(),
          'variants': lambda: make_variants()}


def main(argv=None):
    global REFERENCE
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument('--reference', default=os.environ.get('LM_REFERENCE'),
                    help='path of the reference checkout (or LM_REFERENCE)')
    ap.add_argument('fixtures', nargs='*', choices=[[], *MAKERS],
                    help='fixtures to write (default: all)')
    a = ap.parse_args(argv)
    if not a.reference:
        ap.error('name the reference checkout with --reference or '
                 'LM_REFERENCE')
    REFERENCE = a.reference
    import_reference()
    for name in a.fixtures or list(MAKERS):
        MAKERS[name]()
    print('golden fixtures written to', HERE)


if __name__ == '__main__':
    main()
