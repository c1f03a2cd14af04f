'''Generate the golden fixtures of tests/golden/ by running the reference.

Run from the repository root on a machine that has the reference checkout
(default ``/root/reference``; override with ``LM_REFERENCE``):

    python tests/golden/make_golden.py

The reference package is made importable as ``pylorenzmie`` through a
symlink in a temporary directory, with an empty ``trackpy`` stub (its
analysis/__init__.py imports Localizer, which imports trackpy).  The numpy
FP64 model is imported explicitly from ``pylorenzmie.theory.LorenzMie``
because the package-level ``LorenzMie`` resolves to the fastmath numba
backend (theory/__init__.py:33-38).

Outputs (small, committed):
  ab.npz        Sphere.mie_coefficients for a table of spheres
  layered.npz   sphere_coefficients (one layer, scalar input) for a table
  holo.npz      LorenzMie.field/hologram for the reference tests' geometries
  fit.npz       a seeded 201x201 fit by the reference Optimizer
  estimate.npz  seeded DEEstimator and RadialEstimator searches (81x81 crop)
  variants.npz  AberratedLorenzMie and Dimer holograms
'''
import os
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REFERENCE = os.environ.get('LM_REFERENCE', '/root/reference')


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


def make_layered():
    from pylorenzmie.lib.obsolete.sphere_coefficients import \
        sphere_coefficients
    cases = [(0.75, 1.42, 1.340, 0.447), (1.2, 1.5 + 0.01j, 1.34, 0.447),
             (2.0, 1.6, 1.333, 0.532)]
    out = {'cases': np.array(cases, dtype=complex)}
    for i, (a, n, nm, lam) in enumerate(cases):
        out[f'ab_{i}'] = sphere_coefficients(a, n, nm, lam, resolution=None)
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


if __name__ == '__main__':
    import_reference()
    make_ab()
    make_layered()
    make_holo()
    make_fit()
    make_estimate()
    make_variants()
    print('golden fixtures written to', HERE)
