'''GPU: model variants on the same kernels -- spherical aberration fused
into the field kernel, Cluster / Dimer superposition -- against the
reference's own holograms (tests/golden/variants.npz), and device fits of
aberrated models against the oracle's fit.'''
import numpy as np
import pytest

from oracle import field as ofield

pytestmark = pytest.mark.gpu

KEYS = ('x_p', 'y_p', 'z_p', 'a_p', 'n_p', 'k_p')


def _inst():
    from pylorenzmie_b200 import Instrument
    return Instrument(wavelength=0.447, magnification=0.048, n_m=1.340)


@pytest.mark.parametrize('fp64', [True, False])
def test_aberrated_hologram_matches_reference(golden_variants, fp64):
    from pylorenzmie_b200 import AberratedLorenzMie, Sphere, LorenzMie
    g = golden_variants
    shape = tuple(g['shape'])
    for i in range(2):
        case = g[f'ab_case_{i}']
        s = Sphere(a_p=case[4], n_p=case[5], k_p=case[6])
        s.r_p = case[1:4]
        m = AberratedLorenzMie(coordinates=LorenzMie.meshgrid(shape),
                               particle=s, instrument=_inst(),
                               spherical=case[0], double_precision=fp64)
        ref = g[f'ab_holo_{i}']
        h = m.hologram()
        tol = 1e-10 if fp64 else 2e-5 + 2e-6 * np.abs(ref)
        assert np.all(np.abs(h - ref) <= tol), i
        assert m.properties['spherical'] == case[0]
        assert 'z_p' in m.jac_params and 'spherical' not in m.jac_params
        if not fp64:
            # the analytic Jacobian carries the aberration
            # (lmb_jacobian_aberrated): central differences of the
            # oracle's aberrated hologram
            J = m.jac()
            p = list(case[1:7])
            c = ofield.meshgrid(shape)
            for j, name in enumerate(KEYS):
                h = 1e-4 if j < 5 else 1e-6
                pp, pm = list(p), list(p)
                pp[j] += h
                pm[j] -= h
                fd = (ofield.aberrated_hologram(
                    c, [dict(zip(KEYS, pp))], ofield.DEFAULT_INSTRUMENT,
                    case[0]) - ofield.aberrated_hologram(
                    c, [dict(zip(KEYS, pm))], ofield.DEFAULT_INSTRUMENT,
                    case[0])) / (2 * h)
                err = np.abs(J[name] - fd).max() / np.abs(fd).max()
                assert err < 3e-4, (i, name, err)
    # spherical = 0 is the ideal model, analytic Jacobian included
    m.spherical = 0.
    plain = LorenzMie(coordinates=m.coordinates, particle=s,
                      instrument=_inst(), double_precision=fp64)
    np.testing.assert_array_equal(m.hologram(), plain.hologram())
    assert 'z_p' in m.jac_params


@pytest.mark.parametrize('fp64', [True, False])
def test_dimer_hologram_matches_reference(golden_variants, fp64):
    from pylorenzmie_b200 import Dimer, LorenzMie, Sphere
    g = golden_variants
    x, y, z, a, n, k, theta, phi = g['dimer_case']
    d = Dimer(magnification=0.048)
    d.a_p, d.n_p = a, n
    d.r_p = [x, y, z]
    d.theta, d.phi = theta, phi
    m = LorenzMie(coordinates=LorenzMie.meshgrid(tuple(g['shape'])),
                  particle=d, instrument=_inst(), double_precision=fp64)
    ref = g['dimer_holo']
    tol = 1e-10 if fp64 else 2e-5 + 2e-6 * np.abs(ref)
    assert np.all(np.abs(m.hologram() - ref) <= tol)
    # the same pair as two free spheres in one batch item
    pair = []
    for q in d.particles:
        s = Sphere(a_p=q.a_p, n_p=q.n_p, k_p=q.k_p)
        s.r_p = q.r_p + q.r_0
        pair.append(s)
    hb = m.batch_hologram([pair, [pair[0]]])
    np.testing.assert_allclose(hb[0], m.hologram(), atol=1e-12)


def test_aberrated_device_fit():
    '''With spherical != 0 and fixed (a calibrated instrument), the device
    fit (lmb_fit_batch_aberrated) fits the aberrated model: against the oracle's fit of the same hologram (scipy
    lm on a forward-difference Jacobian of the FP64 aberrated model, as the
    reference's Optimizer does on an AberratedLorenzMie) the parameters
    agree to the fit targets or a third of their uncertainty, it recovers
    the sphere, and optimize_batch (one call or streamed admission) and
    optimize_stream give optimize's result exactly.'''
    from oracle import fit as ofit
    from pylorenzmie_b200 import (AberratedLorenzMie, Sphere, Optimizer,
                                  Hologram, LorenzMie)
    shape = (61, 61)
    truth = dict(zip(KEYS, [30.4, 29.8, 150., 0.75, 1.45, 0.]))
    c = ofield.meshgrid(shape)
    inst = ofield.DEFAULT_INSTRUMENT
    tol = {'x_p': 0.02, 'y_p': 0.02, 'z_p': 0.02, 'a_p': 1e-3, 'n_p': 1e-4}
    for spherical in (1.5, -3.):
        h = ofield.aberrated_hologram(c, [truth], inst, spherical)
        data = h + np.random.default_rng(3).normal(0., 0.05, h.shape)
        start = [30., 30., 158., 0.78, 1.46, 0.]
        s = Sphere(a_p=start[3], n_p=start[4], k_p=0.)
        s.r_p = start[:3]
        m = AberratedLorenzMie(coordinates=LorenzMie.meshgrid(shape),
                               particle=s, instrument=_inst(),
                               spherical=spherical)
        opt = Optimizer(model=m)
        # by default 'spherical' is free too (the reference's default
        # fixed list does not name it): scipy's host loop fits it
        assert 'spherical' in opt.variables and not opt._device_fit_ok()
        # a calibrated instrument: 'spherical' fixed, the device fit
        opt.fixed = opt.fixed + ['spherical']
        assert opt._device_fit_ok()
        holo = Hologram(data.reshape(shape))
        r = opt.optimize(holo)
        assert r['success']
        ref = ofit.fit(data, c, dict(zip(KEYS, start)), inst,
                       spherical=spherical)
        assert ref['success']
        for k in tol:
            bound = max(tol[k], ref['d' + k] / 3.)
            assert abs(r[k] - ref[k]) <= bound, (spherical, k, r[k], ref[k])
        assert abs(r['a_p'] - 0.75) < 0.01 and abs(r['z_p'] - 150.) < 1.
        starts = np.array([start, start])
        df = opt.optimize_batch([holo, holo], starts=starts)
        dfs = next(opt.optimize_stream(iter([([holo, holo], starts)])))
        # streamed admission (the batch in three portions) too
        dfc = opt.optimize_batch([holo] * 3, starts=np.array([start] * 3),
                                 chunks=3)
        for k in tol:
            assert np.all(df[k].to_numpy() == r[k]), k
            assert np.all(dfs[k].to_numpy() == r[k]), k
            assert np.all(dfc[k].to_numpy() == r[k]), k
        # the ideal model fits the aberrated data worse
        s0 = Sphere(a_p=start[3], n_p=start[4], k_p=0.)
        s0.r_p = start[:3]
        plain = Optimizer(model=LorenzMie(coordinates=LorenzMie.meshgrid(
            shape), particle=s0, instrument=_inst()))
        rp = plain.optimize(holo)
        assert rp['redchi'] > r['redchi']


@pytest.mark.parametrize('fp64', [True, False])
def test_aberrated_population_objective(fp64):
    '''The estimators' population objective for an AberratedLorenzMie
    model applies the aberration phase in the same launch: against one
    aberrated model.hologram() per candidate (the reference's objective,
    NaN skipped) to 1e-10 in FP64 and FP32 accuracy otherwise; the
    many-crop form equals the one-crop form exactly.'''
    from pylorenzmie_b200 import AberratedLorenzMie, Sphere, LorenzMie
    from pylorenzmie_b200.analysis._population import (PopulationChi2,
                                                        CropPopulations,
                                                        batchable)
    from pylorenzmie_b200.analysis.DEEstimator import _HostObjective
    rng = np.random.default_rng(12)
    shape = (41, 47)
    c = ofield.meshgrid(shape)
    keep = rng.random(c.shape[1]) < 0.3
    coords = c[:, keep]
    truth = dict(zip(KEYS, [20.4, 23.1, 140., 0.8, 1.45, 0.]))
    data = ofield.aberrated_hologram(coords, [truth], ofield.DEFAULT_INSTRUMENT,
                                     2.) + rng.normal(0., 0.05, coords.shape[1])
    s = Sphere(a_p=0.8, n_p=1.45, k_p=0.)
    s.r_p = [20.4, 23.1, 140.]
    m = AberratedLorenzMie(coordinates=coords, particle=s, instrument=_inst(),
                           spherical=2., double_precision=fp64)
    variables = ['z_p', 'a_p', 'n_p']
    assert batchable(m, variables)
    S = 24
    X = np.vstack([rng.uniform(80., 300., S), rng.uniform(0.4, 2.0, S),
                   rng.uniform(1.35, 1.9, S)])
    got = PopulationChi2(m, data, coords, variables, 0.05)(X)
    ref = _HostObjective(m, data, variables, 0.05)(X)
    np.testing.assert_allclose(got, ref, rtol=1e-10 if fp64 else 2e-5)
    pop = CropPopulations([(m, data, coords, variables)], 0.05)
    np.testing.assert_array_equal(pop.evaluate({0: X})[0], got)
