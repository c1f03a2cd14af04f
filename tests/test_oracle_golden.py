'''Pin the FP64 oracle to the reference: the golden fixtures were produced
by running the reference itself (tests/golden/make_golden.py).'''
import numpy as np
import pytest

from oracle import mie, field, fit

KEYS = ('x_p', 'y_p', 'z_p', 'a_p', 'n_p', 'k_p')


def test_mie_coefficients(golden_ab):
    for i, case in enumerate(golden_ab['cases']):
        ab = mie.mie_coefficients(*case)
        ref = golden_ab[f'ab_{i}']
        assert ab.shape == ref.shape and ab.dtype == np.complex128
        np.testing.assert_array_equal(ab[0], 0j)
        assert np.abs(ab - ref).max() <= 1e-12 * np.abs(ref).max() + 1e-300


def test_wiscombe_yang_pins(golden_ab):
    # the reference's own known answers (tests/test_sphere.py:65-81)
    assert mie.wiscombe_yang(1., 10. + 0.j) == 10
    assert mie.wiscombe_yang(10., 10. + 0.j) == 100
    assert mie.wiscombe_yang(4210., 10. + 0.j) == 42100
    assert mie.neves_pisignano(10.) == 11
    got = [mie.wiscombe_yang(x, m) for x, m in
           zip(golden_ab['wy_x'], golden_ab['wy_m'])]
    assert got == list(golden_ab['wy_n'])
    assert [mie.neves_pisignano(x) for x in golden_ab['np_x']] == \
        list(golden_ab['np_n'])


def test_layered_one_layer(golden_layered):
    for i, (a, n, nm, lam) in enumerate(golden_layered['cases']):
        ab = mie.layered_coefficients([a.real], [n], nm.real, lam.real)
        ref = golden_layered[f'ab_{i}']
        assert ab.shape == ref.shape
        assert np.abs(ab - ref).max() <= 1e-12 * np.abs(ref).max()


def multilayer_cases(golden_layered):
    for i in range(int(golden_layered['multi_count'])):
        nm, lam = golden_layered[f'multi_medium_{i}']
        yield (golden_layered[f'multi_radii_{i}'],
               golden_layered[f'multi_indices_{i}'], nm, lam,
               golden_layered[f'multi_ab_{i}'])


def test_layered_multilayer(golden_layered):
    '''2-, 3- and 4-layer spheres against the reference's own Yang
    recurrences (lib/obsolete/sphere_coefficients.py:126-215, run with its
    input handling repaired by tests/golden/make_golden.py).'''
    n = 0
    for radii, idx, nm, lam, ref in multilayer_cases(golden_layered):
        ab = mie.layered_coefficients(radii, idx, nm, lam)
        assert ab.shape == ref.shape
        assert np.abs(ab - ref).max() <= 1e-12 * np.abs(ref).max()
        n += 1
    assert n >= 8


def test_layered_reduces_to_homogeneous():
    '''Equal indices in every layer: the multilayer recurrence reproduces
    the homogeneous sphere (up to its D1 start one order higher).'''
    for radii in ([0.3, 0.75], [0.2, 0.5, 0.75], [0.5, 1.0, 1.5]):
        n = 1.45 + 0.002j
        ab_l = mie.layered_coefficients(radii, [n] * len(radii), 1.34, 0.447)
        ab_h = mie.mie_coefficients(radii[-1], n.real, n.imag, 1.34, 0.447)
        assert ab_l.shape == ab_h.shape
        assert np.abs(ab_l - ab_h).max() < 1e-6


@pytest.mark.parametrize('name', ['torch64', 'cupy128', 'pair96', 'absorb48',
                                  'below40', 'sph_nb32', 'sph_b32',
                                  'cart_nb32', 'big64'])
def test_hologram_and_field(golden_holo, name):
    shape = tuple(golden_holo[name + '_shape'])
    parts = [dict(zip(KEYS, p)) for p in golden_holo[name + '_particles']]
    cart, bohren = (bool(v) for v in golden_holo[name + '_flags'])
    c = field.meshgrid(shape)
    h = field.hologram(c, parts, field.DEFAULT_INSTRUMENT, cart, bohren)
    np.testing.assert_allclose(h, golden_holo[name + '_holo'], rtol=0,
                               atol=1e-12)
    if name + '_field' in golden_holo:
        f = field.field(c, parts, field.DEFAULT_INSTRUMENT, cart, bohren)
        assert np.abs(f - golden_holo[name + '_field']).max() < 1e-12


def test_fit_matches_reference(golden_fit):
    shape = tuple(golden_fit['shape'])
    start = dict(zip(KEYS, golden_fit['start']))
    r = fit.fit(golden_fit['data'], field.meshgrid(shape), start,
                field.DEFAULT_INSTRUMENT)
    ref = dict(zip(golden_fit['keys'], golden_fit['values']))
    for k, v in ref.items():
        assert abs(float(r[k]) - v) <= 1e-9 * max(1., abs(v)), k
    assert r['nfev'] == int(golden_fit['nfev'])
    assert r['status'] == int(golden_fit['status'])


def test_coordinates_and_wavenumber():
    c = field.coordinates3([[1, 2], [3, 4]])
    assert c.shape == (3, 2) and np.all(c[2] == 0)
    with pytest.raises(ValueError):
        field.coordinates3(np.zeros((4, 2)))
    k = field.wavenumber(1.34, 0.447, 0.048)
    assert abs(k - 2 * np.pi / 0.447 * 1.34 * 0.048) < 1e-15


def test_oracle_estimators_match_reference(golden_estimate):
    '''The oracle's DEEstimator and RadialEstimator restatements reproduce
    the reference's seeded searches (same pixel subset, same scipy DE
    trajectory).'''
    from oracle import estimate, field
    g = golden_estimate
    data = g['data']
    coords = field.meshgrid(data.shape, flatten=False)
    part = dict(zip(('x_p', 'y_p', 'z_p', 'a_p', 'n_p', 'k_p'),
                    [0., 0., 100., 1.0, 1.5, 0.]))
    np.random.seed(int(g['mask_seed']))
    p, _ = estimate.de_estimate(data, coords, part, field.DEFAULT_INSTRUMENT,
                                seed=int(g['de_seed']))
    got = np.array([p[k] for k in ('x_p', 'y_p', 'z_p', 'a_p', 'n_p')])
    np.testing.assert_allclose(got, g['de'][:5], rtol=1e-9)
    p, _ = estimate.radial_estimate(data, coords, (0., 0.), part,
                                    field.DEFAULT_INSTRUMENT,
                                    seed=int(g['de_seed']))
    got = np.array([p[k] for k in ('x_p', 'y_p', 'z_p', 'a_p', 'n_p')])
    np.testing.assert_allclose(got, g['radial'][:5], rtol=1e-9)


def test_oracle_aberrated_and_dimer(golden_variants):
    '''Aberrated holograms and a Dimer (two spheres placed by the cluster
    geometry) against the reference's own output.'''
    g = golden_variants
    shape = tuple(g['shape'])
    c = field.meshgrid(shape)
    keys = ('x_p', 'y_p', 'z_p', 'a_p', 'n_p', 'k_p')
    for i in range(2):
        case = g[f'ab_case_{i}']
        h = field.aberrated_hologram(c, [dict(zip(keys, case[1:]))],
                                     field.DEFAULT_INSTRUMENT, case[0])
        assert np.abs(h - g[f'ab_holo_{i}']).max() < 1e-10
    h = field.hologram(c, [dict(zip(keys, s)) for s in g['dimer_spheres']],
                       field.DEFAULT_INSTRUMENT)
    assert np.abs(h - g['dimer_holo']).max() < 1e-10


def test_cluster_and_dimer_geometry(golden_variants):
    '''Host classes: the Dimer places its spheres where the reference does;
    moving a Cluster moves its members' origins.'''
    from pylorenzmie_b200 import Dimer, Cluster, Sphere
    g = golden_variants
    x, y, z, a, n, k, theta, phi = g['dimer_case']
    d = Dimer(magnification=0.048)
    d.a_p = a
    d.n_p = n
    d.r_p = [x, y, z]
    d.theta = theta
    d.phi = phi
    got = np.array([[*(q.r_p + q.r_0), q.a_p, q.n_p, q.k_p]
                    for q in d.particles])
    np.testing.assert_allclose(got, g['dimer_spheres'], rtol=1e-13)
    assert set(d.properties) == {'x_p', 'y_p', 'z_p', 'a_p', 'n_p', 'k_p',
                                 'theta', 'phi'}
    s1, s2 = Sphere(), Sphere()
    s2.r_p = [5., 0., 0.]
    cl = Cluster(particles=[s1, s2])
    cl.r_p = [10., 20., 100.]
    assert list(s2.r_p + s2.r_0) == [15., 20., 100.]
    assert len(cl) == 2 and list(cl)[1] is s2
