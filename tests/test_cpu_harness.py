'''The kernels' own arithmetic, compiled for the CPU (tests/cpu_harness),
against the FP64 oracle and scipy.

This checks, without a GPU, the exact code the sm_100a kernels run: the
FP64 Mie recurrences with tangents, the per-pixel sums in FP32 and FP64,
the forward-mode Jacobian, and the Levenberg-Marquardt state machine
(restated MINPACK lmder) against scipy's least_squares(method='lm').
'''
import ctypes

import numpy as np
import pytest
from scipy.optimize import least_squares

from oracle import mie, field, fit
from tests.cpu_harness.loader import Harness, ptr

KEYS = ('x_p', 'y_p', 'z_p', 'a_p', 'n_p', 'k_p')
K = field.wavenumber(1.34, 0.447, 0.048)


@pytest.fixture(scope='module')
def h():
    return Harness()


def test_sphere_ab_and_tangents(h, golden_ab):
    for i, case in enumerate(golden_ab['cases']):
        ab, dab = h.sphere_ab(*case, deriv=True)
        ref = golden_ab[f'ab_{i}']
        assert ab.shape == ref.shape
        assert np.abs(ab - ref).max() <= 1e-12 * np.abs(ref).max() + 1e-300
    # tangents against central differences of the oracle
    for (a, n, k) in [(0.75, 1.45, 0.), (1.5, 1.59, 0.002), (0.4, 1.38, 0.)]:
        ab, dab = h.sphere_ab(a, n, k, 1.34, 0.447, deriv=True)
        da, dn = 1e-6 * a, 1e-6
        fa = (mie.mie_coefficients(a + da, n, k, 1.34, 0.447) -
              mie.mie_coefficients(a - da, n, k, 1.34, 0.447)) / (2 * da)
        fn = (mie.mie_coefficients(a, n + dn, k, 1.34, 0.447) -
              mie.mie_coefficients(a, n - dn, k, 1.34, 0.447)) / (2 * dn)
        assert np.abs(dab[:, :2] - fa).max() < 1e-6 * np.abs(fa).max()
        assert np.abs(dab[:, 2:] - fn).max() < 1e-6 * np.abs(fn).max()


@pytest.mark.parametrize('name', ['torch64', 'cupy128', 'pair96', 'absorb48',
                                  'below40', 'sph_nb32', 'sph_b32',
                                  'cart_nb32', 'big64'])
@pytest.mark.parametrize('fp64', [0, 1])
def test_pixel_sums(h, golden_holo, name, fp64):
    shape = tuple(golden_holo[name + '_shape'])
    cart, bohren = (bool(v) for v in golden_holo[name + '_flags'])
    c = field.coordinates3(field.meshgrid(shape))
    E = np.zeros((3, c.shape[1]), complex)
    for p in golden_holo[name + '_particles']:
        ab = h.sphere_ab(p[3], p[4], p[5], 1.34, 0.447)
        E += h.field(c, p[:3], ab, K, cart, bohren, fp64)
    holo = np.sum(np.abs(E + np.array([[1], [0], [0]])) ** 2, axis=0)
    err = np.abs(holo - golden_holo[name + '_holo']).max()
    assert err <= (1e-11 if fp64 else 2e-5), err
    if name + '_field' in golden_holo:
        ferr = np.abs(E - golden_holo[name + '_field']).max()
        assert ferr <= (1e-11 if fp64 else 2e-5), ferr


@pytest.mark.parametrize('shape,p', [
    ((48, 48), [20.3, 25.7, 120., 0.9, 1.6, 0.01]),
    ((40, 40), [20., 20., -130., 0.6, 1.5, 0.]),
    ((33, 33), [16., 16., 80., 1.0, 1.4, 0.]),
])
@pytest.mark.parametrize('fp64', [0, 1])
def test_jacobian(h, shape, p, fp64):
    c = field.coordinates3(field.meshgrid(shape))
    ab, dab = h.sphere_ab(p[3], p[4], p[5], 1.34, 0.447, deriv=True)
    H, J = h.jacobian(c, p[:3], ab, dab, K, True, fp64)
    inst = field.DEFAULT_INSTRUMENT
    h0 = field.hologram(c, [dict(zip(KEYS, p))], inst)
    assert np.abs(H - h0).max() < (1e-11 if fp64 else 2e-5)
    for j in range(6):
        step = 1e-5 * max(abs(p[j]), 1e-2) if j < 5 else 1e-7
        pp, pm = list(p), list(p)
        pp[j] += step
        pm[j] -= step
        fd = (field.hologram(c, [dict(zip(KEYS, pp))], inst) -
              field.hologram(c, [dict(zip(KEYS, pm))], inst)) / (2 * step)
        err = np.abs(J[j] - fd).max() / np.abs(fd).max()
        assert err < (1e-5 if fp64 else 3e-4), (KEYS[j], err)


def _lm_run(h, model, data, variables, p0, noise=0.05):
    lib = h.lib
    slots = np.array(variables, dtype=np.int32)
    x0 = np.array([p0[j] for j in variables])
    hd = lib.h_lm_new(len(variables), ptr(slots, ctypes.POINTER(ctypes.c_int)),
                      ptr(x0), 1e-4, 1e-6, 1e-6, 100., 2000)
    p = np.array(p0, float)
    xn = np.zeros(6)
    while True:
        H, J = model(p)
        r = (H - data) / noise
        Jn = J / noise
        jtj = np.array([Jn[a] @ Jn[b] for a in range(6) for b in range(a, 6)])
        done = lib.h_lm_feed(hd, float(r @ r), ptr(jtj),
                             ptr(np.ascontiguousarray(Jn @ r)), ptr(xn))
        if done:
            break
        p = np.array(p0, float)
        for a, j in enumerate(variables):
            p[j] = xn[a]
    x = np.zeros(6)
    info, nfev, njev = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    rc, dp = ctypes.c_double(), np.zeros(6)
    lib.h_lm_result(hd, data.size, ptr(x), ctypes.byref(info),
                    ctypes.byref(nfev), ctypes.byref(njev), ctypes.byref(rc),
                    ptr(dp))
    lib.h_lm_free(hd)
    n = len(variables)
    return x[:n], info.value, nfev.value, njev.value, rc.value, dp[:n]


@pytest.mark.parametrize('variables', [[0, 1, 2, 3, 4], [0, 1, 2, 3, 4, 5],
                                       [2, 3, 4], [3, 4]])
def test_lm_state_machine_matches_scipy(h, golden_fit, variables):
    '''Same residuals and Jacobian in, same iterates out: the device LM
    logic follows MINPACK lmder as scipy runs it.'''
    shape = tuple(golden_fit['shape'])
    c = field.coordinates3(field.meshgrid(shape))
    data = golden_fit['data']
    start = golden_fit['start']

    def model(p):
        ab, dab = h.sphere_ab(p[3], p[4], p[5], 1.34, 0.447, deriv=True)
        return h.jacobian(c, p[:3], ab, dab, K, True, 1)

    x, info, nfev, njev, redchi, dp = _lm_run(h, model, data, variables,
                                              start)
    base = np.array(start, float)

    def params(v):
        q = base.copy()
        q[variables] = v
        return q
    res = least_squares(lambda v: (model(params(v))[0] - data) / 0.05,
                        base[variables],
                        jac=lambda v: model(params(v))[1][variables].T / 0.05,
                        method='lm', ftol=1e-4, xtol=1e-6, gtol=1e-6,
                        max_nfev=2000, x_scale='jac')
    rc, sdp = fit.statistics(res, data.size)
    np.testing.assert_allclose(x, res.x, rtol=1e-9, atol=1e-9)
    assert nfev == res.nfev and njev == res.njev
    assert {1: 2, 2: 3, 3: 4, 4: 1}[info] == res.status
    assert abs(redchi - rc) < 1e-9 * rc
    np.testing.assert_allclose(dp, sdp, rtol=1e-6)


@pytest.mark.parametrize('spherical', [0.9, -2.5])
def test_aberrated_jacobian(h, spherical):
    '''The aberrated epilogue of the device fits: the hologram equals the
    oracle's AberratedLorenzMie hologram, and the six columns equal central
    differences of it (FP64 sums; FP32 sums within FP32 accuracy).'''
    inst = field.DEFAULT_INSTRUMENT
    c = field.coordinates3(field.meshgrid((41, 53)))
    p = np.array([20.3, 25.1, 120., 0.8, 1.45, 0.002])
    caber = 4. * inst['n_m'] ** 3 / K * spherical
    ab, dab = h.sphere_ab(p[3], p[4], p[5], 1.34, 0.447, deriv=True)
    H, J = h.jacobian_aberrated(c, p[:3], ab, dab, K, caber, fp64=True)

    def holo(q):
        return field.aberrated_hologram(c, [dict(zip(KEYS, q))], inst,
                                        spherical)
    ref = holo(p)
    np.testing.assert_allclose(H, ref, rtol=1e-10, atol=1e-12)
    steps = [1e-4, 1e-4, 1e-3, 1e-6, 1e-6, 1e-6]
    for j, dj in enumerate(steps):
        qp, qm = p.copy(), p.copy()
        qp[j] += dj
        qm[j] -= dj
        fd = (holo(qp) - holo(qm)) / (2 * dj)
        scale = np.abs(fd).max()
        assert np.abs(J[j] - fd).max() <= 2e-5 * scale, \
            (KEYS[j], np.abs(J[j] - fd).max() / scale)
    H32, J32 = h.jacobian_aberrated(c, p[:3], ab, dab, K, caber, fp64=False)
    assert np.all(np.abs(H32 - H) <= 2e-5 * (1 + np.abs(H)))
    for j in range(6):
        scale = np.abs(J[j]).max()
        assert np.abs(J32[j] - J[j]).max() <= 2e-4 * scale, KEYS[j]
    # no aberration: the ideal epilogue exactly
    H0, J0 = h.jacobian_aberrated(c, p[:3], ab, dab, K, 0., fp64=True)
    H1, J1 = h.jacobian_rev(c, p[:3], ab, dab, K, fp64=True)
    np.testing.assert_array_equal(H0, H1)
    np.testing.assert_array_equal(J0, J1)


@pytest.mark.parametrize('radii,idx', [
    ([0.3, 0.75], [1.6, 1.45 + 0.002j]),
    ([0.4, 0.8, 1.2], [1.8 + 0.01j, 1.33, 1.5]),
    ([0.5, 1.2, 2.0], [1.4, 1.7, 1.55 + 0.001j]),
])
def test_layered_ab_and_tangents(h, radii, idx):
    ab, dab = h.layered_ab(radii, idx, 1.34, 0.447, deriv=True)
    ref = mie.layered_coefficients(radii, idx, 1.34, 0.447)
    assert ab.shape == ref.shape
    assert np.abs(ab - ref).max() <= 1e-12 * np.abs(ref).max()
    ap = radii[-1]
    frac = np.asarray(radii) / ap
    da = 1e-6 * ap
    fa = (mie.layered_coefficients(frac * (ap + da), idx, 1.34, 0.447) -
          mie.layered_coefficients(frac * (ap - da), idx, 1.34, 0.447)) / (2 * da)
    ip, im = list(idx), list(idx)
    ip[-1] += 1e-6
    im[-1] -= 1e-6
    fn = (mie.layered_coefficients(radii, ip, 1.34, 0.447) -
          mie.layered_coefficients(radii, im, 1.34, 0.447)) / 2e-6
    assert np.abs(dab[:, :2] - fa).max() < 1e-6 * np.abs(fa).max()
    assert np.abs(dab[:, 2:] - fn).max() < 1e-6 * np.abs(fn).max()


def test_layered_one_layer_matches_reference(h, golden_layered):
    for i, (a, n, nm, lam) in enumerate(golden_layered['cases']):
        ab = h.layered_ab([a.real], [n], nm.real, lam.real)
        ref = golden_layered[f'ab_{i}']
        assert np.abs(ab - ref).max() <= 1e-12 * np.abs(ref).max()


def test_layered_multilayer_matches_reference(h, golden_layered):
    '''The kernels' Yang recurrences (both the serial and the split shell
    forms) against the reference's own 2-4 layer coefficients.'''
    from tests.test_oracle_golden import multilayer_cases
    for radii, idx, nm, lam, ref in multilayer_cases(golden_layered):
        for split in (False, True):
            ab = h.layered_ab(radii, idx, nm, lam, split=split)
            assert ab.shape == ref.shape
            assert np.abs(ab - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize('shape,p', [
    ((48, 48), [20.3, 25.7, 120., 0.9, 1.6, 0.01]),
    ((40, 40), [20., 20., -130., 0.6, 1.5, 0.]),
    ((33, 33), [16., 16., 80., 1.0, 1.4, 0.]),
    ((21, 31), [15.2, 10.1, 60., 2.5, 1.7, 0.002]),
])
def test_jacobian_pair_loop(h, shape, p):
    '''The packed two-pixel loop (signed recurrences, pair records) gives the
    scalar loop's hologram and Jacobian to FP32 rounding, and the FD
    Jacobian of the oracle to the scalar loop's tolerance.'''
    c = field.coordinates3(field.meshgrid(shape))
    ab, dab = h.sphere_ab(p[3], p[4], p[5], 1.34, 0.447, deriv=True)
    H1, J1 = h.jacobian(c, p[:3], ab, dab, K, True, 0)
    H2, J2 = h.jacobian_pair(c, p[:3], ab, dab, K, True)
    # FP32 rounding differs in order only: relative to the hologram's size
    assert np.all(np.abs(H2 - H1) < 1e-5 + 4e-6 * np.abs(H1))
    for j in range(6):
        scale = np.abs(J1[j]).max()
        assert np.abs(J2[j] - J1[j]).max() < 1e-4 * scale, KEYS[j]
    inst = field.DEFAULT_INSTRUMENT
    h0 = field.hologram(c, [dict(zip(KEYS, p))], inst)
    assert np.all(np.abs(H2 - h0) < 2e-5 + 2e-6 * np.abs(h0))
    for j in range(6):
        step = 1e-5 * max(abs(p[j]), 1e-2) if j < 5 else 1e-7
        pp, pm = list(p), list(p)
        pp[j] += step
        pm[j] -= step
        fd = (field.hologram(c, [dict(zip(KEYS, pp))], inst) -
              field.hologram(c, [dict(zip(KEYS, pm))], inst)) / (2 * step)
        err = np.abs(J2[j] - fd).max() / np.abs(fd).max()
        assert err < 3e-4, (KEYS[j], err)


@pytest.mark.parametrize('name', ['torch64', 'cupy128', 'pair96', 'absorb48',
                                  'below40', 'sph_nb32', 'sph_b32',
                                  'cart_nb32', 'big64'])
def test_pixel_sums_pair_loop(h, golden_holo, name):
    '''The packed two-pixel value loop (the FP32 field/hologram kernel)
    against the reference's own fields and holograms.'''
    shape = tuple(golden_holo[name + '_shape'])
    cart, bohren = (bool(v) for v in golden_holo[name + '_flags'])
    c = field.coordinates3(field.meshgrid(shape))
    E = np.zeros((3, c.shape[1]), complex)
    for p in golden_holo[name + '_particles']:
        ab = h.sphere_ab(p[3], p[4], p[5], 1.34, 0.447)
        E += h.field_pair(c, p[:3], ab, K, cart, bohren)
    holo = np.sum(np.abs(E + np.array([[1], [0], [0]])) ** 2, axis=0)
    ref = golden_holo[name + '_holo']
    assert np.all(np.abs(holo - ref) <= 2e-5 + 2e-6 * np.abs(ref))
    if name + '_field' in golden_holo:
        assert np.abs(E - golden_holo[name + '_field']).max() <= 2e-5


@pytest.mark.parametrize('shape,p', [
    ((48, 48), [20.3, 25.7, 120., 0.9, 1.6, 0.01]),
    ((40, 40), [20., 20., -130., 0.6, 1.5, 0.]),
    ((33, 33), [16., 16., 80., 1.0, 1.4, 0.]),
    ((21, 31), [15.2, 10.1, 60., 2.5, 1.7, 0.002]),
])
@pytest.mark.parametrize('bohren', [True, False])
def test_reverse_epilogue_matches_forward(h, shape, p, bohren):
    '''The reverse-mode epilogue gives the forward-mode (dual-number)
    epilogue's hologram and Jacobian: to FP64 rounding in FP64, to FP32
    rounding in FP32 (on-axis pixels included: the grids contain x_p, y_p
    in the first three cases).'''
    c = field.coordinates3(field.meshgrid(shape))
    ab, dab = h.sphere_ab(p[3], p[4], p[5], 1.34, 0.447, deriv=True)
    for fp64, rtol in ((1, 1e-10), (0, 2e-5)):
        H1, J1 = h.jacobian(c, p[:3], ab, dab, K, bohren, fp64)
        H2, J2 = h.jacobian_rev(c, p[:3], ab, dab, K, bohren, fp64)
        assert np.all(np.abs(H2 - H1) <= rtol * (1 + np.abs(H1)))
        for j in range(6):
            scale = np.abs(J1[j]).max() + 1e-30
            assert np.abs(J2[j] - J1[j]).max() <= 10 * rtol * scale, \
                (KEYS[j], fp64, np.abs(J2[j] - J1[j]).max() / scale)


@pytest.mark.parametrize('radii,idx', [
    ([0.3, 0.75], [1.6, 1.45 + 0.002j]),
    ([0.4, 0.8, 1.2], [1.8 + 0.01j, 1.33, 1.5]),
    ([0.5, 1.2, 2.0], [1.4, 1.7, 1.55 + 0.001j]),
    ([0.2, 0.5, 0.9, 1.4, 2.4], [1.35, 1.7, 1.4, 1.6 + 0.003j, 1.5]),
])
def test_layered_split_shell_matches_serial(h, radii, idx):
    '''The split shell functions of the warp-parallel kernel path (each
    argument's D3 chain stored, Q's factors per order and their running
    product, then independent per-order updates) agree with the fused
    serial pass to rounding: Q's factors are grouped differently, so the
    two differ by ~1e-15 of the largest coefficient (1e-13 asserted).'''
    a1, d1 = h.layered_ab(radii, idx, 1.34, 0.447, deriv=True)
    a2, d2 = h.layered_ab(radii, idx, 1.34, 0.447, deriv=True, split=True)
    assert np.abs(a2 - a1).max() <= 1e-13 * np.abs(a1).max()
    assert np.abs(d2 - d1).max() <= 1e-13 * np.abs(d1).max()


def test_hologram_error_bound(h):
    '''The per-pixel error bound of the FP32 hologram kernel.  A 3 um sphere
    10 px above its top focuses light to H ~ 60 on its axis, where FP32
    is off by more than 2e-5; the bound must cover the FP32 error at every
    pixel, mark those pixels for the FP64 sum, and leave the others within
    2e-5.'''
    P = np.array([[80.3, 79.6, 72.5, 3.0, 1.56, 0.],
                  [20.2, 150.7, 200., 1.5, 1.50, 1e-3],
                  [150.1, 10.4, 130., 2.5, 1.65, 0.]])
    c = field.meshgrid((160, 160))
    ref = field.hologram(c, [dict(zip(KEYS, p)) for p in P],
                         field.DEFAULT_INSTRUMENT)
    h32, terms = h.hologram_pair(field.coordinates3(c), P, K, flag=False)
    err = np.abs(h32.astype(float) - ref)
    assert err.max() > 2e-5        # FP32 alone misses the tolerance here
    bound = 3e-6 * terms[0].astype(float) + 1e-7 * terms[1]
    assert np.all(err <= 0.75 * bound)
    marked, _ = h.hologram_pair(field.coordinates3(c), P, K)
    flag = marked < 0
    assert np.all(flag[bound > 2e-5 * (1 + 1e-4)])
    assert not np.any(flag[bound < 2e-5 * (1 - 1e-4)])
    assert np.all(marked[~flag] == h32[~flag])
    assert np.all(err[~flag] <= 2e-5)
    # the window is centred on the focus; over whole frames about 0.5 %
    assert flag.any() and flag.mean() < 0.25
