'''GPU parity of the generative model: Mie coefficients, field, hologram,
batch API and the analytic Jacobian, through the C-ABI library, against the
reference's golden outputs (tests/golden, made by running the reference)
and the FP64 oracle.

Tolerances: FP64 sums agree with the reference to 1e-11 (absolute, values
of order 1); FP32 sums (the default) to 2e-5 absolute, the hologram error
budget of the FP32+FP64-coefficient method; the Jacobian to 3e-4 of its
column maximum against central finite differences of the FP64 oracle (the
tolerance of the reference's Jacobian test, tests/test_jaxlorenzmie.py:79-101).
'''
import numpy as np
import pytest

from oracle import field as ofield

pytestmark = pytest.mark.gpu

NAMES = ('x_p', 'y_p', 'z_p', 'a_p', 'n_p', 'k_p')
HOLO_CASES = ['torch64', 'cupy128', 'pair96', 'absorb48', 'below40',
              'sph_nb32', 'sph_b32', 'cart_nb32', 'big64']


def spheres_of(P):
    from pylorenzmie_b200 import Sphere
    out = []
    for p in P:
        s = Sphere(a_p=p[3], n_p=p[4], k_p=p[5])
        s.r_p = [p[0], p[1], p[2]]
        out.append(s)
    return out


def model_for(golden, name, fp64=False):
    from pylorenzmie_b200 import LorenzMie, Instrument
    shape = tuple(golden[name + '_shape'])
    inst = Instrument(wavelength=0.447, magnification=0.048, n_m=1.340)
    m = LorenzMie(coordinates=LorenzMie.meshgrid(shape),
                  particle=spheres_of(golden[name + '_particles']),
                  instrument=inst, double_precision=fp64)
    cart, bohren = (bool(v) for v in golden[name + '_flags'])
    return m, cart, bohren


def test_sphere_ab_matches_reference(golden_ab):
    from pylorenzmie_b200 import Sphere
    for i, (a, n, k, nm, lam) in enumerate(golden_ab['cases']):
        ab = Sphere.mie_coefficients(a, n, k, nm, lam)
        ref = golden_ab[f'ab_{i}']
        assert ab.shape == ref.shape
        assert ab.dtype == np.complex128
        np.testing.assert_array_equal(ab[0], 0j)
        err = np.abs(ab - ref).max() / np.abs(ref).max()
        assert err < 1e-11, (i, err)


def test_sphere_ab_large_spheres_vs_oracle():
    '''Spheres of 64..421 orders (the estimators' bounds reach a_p = 10 um
    with n_p = 3), where the medium's D1 is formed by the warp scan: a_n,
    b_n against the oracle's serial recurrences to 1e-11 of their largest
    value, and the a_p / n_p derivatives against central differences of
    the oracle to 1e-6 of their largest value plus the differences' own
    error (steps h and h/2: sharp resonances of lossless spheres).'''
    import torch
    from oracle import mie as omie
    from pylorenzmie_b200.theory import _kernels as K
    rng = np.random.default_rng(17)
    n_m, lam = 1.34, 0.447
    cases = [(10., 3., 0.), (10., 1.0, 0.), (2.6, 1.7, 1e-3), (6., 2.,
                                                                0.), (4., 1.2, 0.)]
    cases += [(rng.uniform(2.8, 10.), rng.uniform(1.0, 3.0),
               rng.choice([0., 0.02])) for _ in range(11)]
    P = np.zeros((len(cases), 6))
    P[:, 3:] = cases
    refs = [omie.mie_coefficients(a, n, k, n_m, lam) for a, n, k in cases]
    nmaxs = [len(r) - 1 for r in refs]
    assert min(nmaxs) >= 64 and max(nmaxs) >= 400
    cap = max(nmaxs)
    ab, dab, nmax = K.sphere_ab(torch.as_tensor(P, device='cuda:0'), n_m,
                                lam, cap, deriv=True)
    ab = ab.cpu().numpy().view(np.complex128)[..., 0]
    dab = dab.cpu().numpy().view(np.complex128)[..., 0]
    np.testing.assert_array_equal(nmax.cpu().numpy(), nmaxs)
    for i, (a, n, k) in enumerate(cases):
        ref = refs[i]
        nm = nmaxs[i]
        err = np.abs(ab[i, :nm + 1] - ref).max() / np.abs(ref).max()
        assert err < 1e-11, (cases[i], err)
        assert np.all(ab[i, nm + 1:] == 0)
        for j, (da, dn) in enumerate(((1e-6, 0.), (0., 1e-7))):
            fds = []
            for f in (1., 0.5):
                up = omie.mie_coefficients(a + f * da, n + f * dn, k, n_m,
                                           lam)
                lo = omie.mie_coefficients(a - f * da, n - f * dn, k, n_m,
                                           lam)
                L = min(len(up), len(lo), nm + 1)
                fds.append((up[:L] - lo[:L]) / (2 * f * (da + dn)))
            L = min(len(fds[0]), len(fds[1]))
            fd = fds[1][:L]
            allowed = 1e-6 * np.abs(fd).max() + 4. * np.abs(fds[0][:L] - fd)
            got = dab[i, :L, 2 * j:2 * j + 2]
            assert np.all(np.abs(got - fd) <= allowed), (cases[i], j)


@pytest.mark.parametrize('name', HOLO_CASES)
def test_hologram_fp32(golden_holo, name):
    m, cart, bohren = model_for(golden_holo, name)
    h = m.hologram(cartesian=cart, bohren=bohren)
    assert h.dtype == np.float64 and h.shape == golden_holo[name + '_holo'].shape
    err = np.abs(h - golden_holo[name + '_holo']).max()
    assert err <= 2e-5, err


@pytest.mark.parametrize('name', HOLO_CASES)
def test_hologram_fp64(golden_holo, name):
    m, cart, bohren = model_for(golden_holo, name, fp64=True)
    h = m.hologram(cartesian=cart, bohren=bohren)
    err = np.abs(h - golden_holo[name + '_holo']).max()
    assert err <= 1e-11, err


@pytest.mark.parametrize('name', [n for n in HOLO_CASES
                                  if n not in ('cupy128', 'pair96')])
@pytest.mark.parametrize('fp64', [False, True])
def test_field(golden_holo, name, fp64):
    m, cart, bohren = model_for(golden_holo, name, fp64)
    f = m.field(cartesian=cart, bohren=bohren)
    assert f.shape == golden_holo[name + '_field'].shape
    err = np.abs(f - golden_holo[name + '_field']).max()
    assert err <= (1e-11 if fp64 else 2e-5), err


def test_reference_backend_tolerances(golden_holo):
    '''The cross-backend pins of the reference's own tests.'''
    m, _, _ = model_for(golden_holo, 'torch64')
    np.testing.assert_allclose(m.hologram(), golden_holo['torch64_holo'],
                               rtol=1e-4, atol=1e-6)
    m, _, _ = model_for(golden_holo, 'cupy128')
    assert np.allclose(m.hologram(), golden_holo['cupy128_holo'], rtol=1e-5)


def test_batch_matches_sequential():
    from pylorenzmie_b200 import LorenzMie, Sphere

    def sphere(x, y, z, a, n):
        s = Sphere(a_p=a, n_p=n)
        s.r_p = [x, y, z]
        return s
    lists = [[sphere(16., 16., 150., 0.75, 1.45)],
             [sphere(10., 20., 200., 1.0, 1.40)],
             [sphere(20., 10., 100., 0.5, 1.50), sphere(24., 24., 180., 0.8, 1.42)],
             []]
    m = LorenzMie(coordinates=LorenzMie.meshgrid((32, 32)))
    hb = m.batch_hologram(lists)
    assert hb.shape == (4, 32 * 32) and hb.dtype == np.float64
    for i, pl in enumerate(lists):
        m.particle = pl if pl else [sphere(0., 0., 100., 0.5, 1.5)]
        if not pl:
            np.testing.assert_allclose(hb[i], 1.0)
            continue
        np.testing.assert_allclose(hb[i], m.hologram(), rtol=1e-5, atol=1e-7)
    fb = m.batch_field(lists)
    assert tuple(fb.shape) == (4, 3, 32 * 32)


@pytest.mark.parametrize('shape,p', [
    ((64, 64), [32., 32., 150., 0.75, 1.45, 0.0]),
    ((48, 48), [20.3, 25.7, 120., 0.9, 1.6, 0.01]),
    ((40, 40), [20., 20., -130., 0.6, 1.5, 0.0]),
    ((33, 33), [16., 16., 80., 1.0, 1.4, 0.0]),
])
def test_jacobian_vs_finite_differences(shape, p):
    from pylorenzmie_b200 import LorenzMie, Sphere
    s = Sphere(a_p=p[3], n_p=p[4], k_p=p[5])
    s.r_p = p[:3]
    m = LorenzMie(coordinates=LorenzMie.meshgrid(shape), particle=s)
    J = m.jac()
    assert set(J) == set(NAMES)
    c = ofield.meshgrid(shape)
    inst = ofield.DEFAULT_INSTRUMENT
    for j, name in enumerate(NAMES):
        h = 1e-4 if j < 5 else 1e-6
        pp, pm = list(p), list(p)
        pp[j] += h
        pm[j] -= h
        fd = (ofield.hologram(c, [dict(zip(NAMES, pp))], inst) -
              ofield.hologram(c, [dict(zip(NAMES, pm))], inst)) / (2 * h)
        assert J[name].dtype == np.float64 and np.all(np.isfinite(J[name]))
        err = np.abs(J[name] - fd).max() / np.abs(fd).max()
        assert err < 3e-4, (name, err)


def test_jac_rejects_multiple_particles():
    from pylorenzmie_b200 import LorenzMie, Sphere
    m = LorenzMie(coordinates=LorenzMie.meshgrid((8, 8)),
                  particle=[Sphere(), Sphere()])
    with pytest.raises(TypeError):
        m.jac()


def test_nmax_above_limit_raises():
    from pylorenzmie_b200 import LorenzMie, Sphere
    m = LorenzMie(coordinates=LorenzMie.meshgrid((8, 8)),
                  particle=Sphere(a_p=100., n_p=1.5))
    with pytest.raises(ValueError):
        m.hologram()
