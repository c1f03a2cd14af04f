'''GPU parity of the device Levenberg-Marquardt fit against the reference.

The reference fit (tests/golden/fit.npz) is the reference Optimizer run on
a seeded 201x201 hologram (config: a_p=0.75 um, n_p=1.42, z_p=200 px,
noise 0.05, start perturbed by 5 % in a_p, 0.02 in n_p, 10 px in z_p).
The device fit must land within a_p 1 nm, n_p 1e-4, z_p 0.02 px (and
x_p, y_p 0.02 px) of it.
'''
import numpy as np
import pandas as pd
import pytest

from oracle import field as ofield, fit as ofit

pytestmark = pytest.mark.gpu

KEYS = ('x_p', 'y_p', 'z_p', 'a_p', 'n_p', 'k_p')
TOL = {'x_p': 0.02, 'y_p': 0.02, 'z_p': 0.02, 'a_p': 1e-3, 'n_p': 1e-4,
       'k_p': 1e-4}


def make_optimizer(start, shape):
    from pylorenzmie_b200 import LorenzMie, Optimizer, Instrument, Sphere
    inst = Instrument(wavelength=0.447, magnification=0.048, n_m=1.340)
    s = Sphere(a_p=start[3], n_p=start[4], k_p=start[5])
    s.r_p = start[:3]
    model = LorenzMie(coordinates=LorenzMie.meshgrid(shape), particle=s,
                      instrument=inst)
    return Optimizer(model=model)


def test_fit_matches_reference(golden_fit):
    from pylorenzmie_b200 import Hologram
    shape = tuple(golden_fit['shape'])
    opt = make_optimizer(golden_fit['start'], shape)
    result = opt.optimize(Hologram(golden_fit['data'].reshape(shape)))
    ref = dict(zip(golden_fit['keys'], golden_fit['values']))
    assert isinstance(result, pd.Series)
    assert list(result.index) == list(golden_fit['keys'])
    assert bool(result['success'])
    assert result['npix'] == shape[0] * shape[1]
    for k in ('x_p', 'y_p', 'z_p', 'a_p', 'n_p'):
        assert abs(result[k] - ref[k]) <= TOL[k], (k, result[k], ref[k])
        assert abs(result['d' + k] / ref['d' + k] - 1) < 1e-2, k
    assert abs(result['redchi'] / ref['redchi'] - 1) < 1e-4
    assert opt._result.nfev == int(golden_fit['nfev'])
    assert opt._result.status == int(golden_fit['status'])
    # the model is left at the fitted values
    assert abs(opt.model.particle.a_p - result['a_p']) < 1e-12
    assert 'a_p' in opt.report()


def _render(seed, shape, p):
    rng = np.random.default_rng(seed)
    c = ofield.meshgrid(shape)
    h = ofield.hologram(c, [dict(zip(KEYS, p))], ofield.DEFAULT_INSTRUMENT)
    return h + rng.normal(0., 0.05, h.shape)


def test_fit_batch_matches_oracle():
    '''16 features of mixed crop sizes in one device call vs the oracle fit
    (the reference algorithm, scipy lm + FD Jacobian) of each.'''
    from pylorenzmie_b200 import Hologram
    rng = np.random.default_rng(7)
    holos, starts, oracle = [], [], []
    for i in range(16):
        s = int(rng.choice([41, 61, 81, 101]))
        c = (s - 1) / 2.
        truth = [c + rng.uniform(-2, 2), c + rng.uniform(-2, 2),
                 rng.uniform(150., 250.), rng.uniform(0.5, 1.0),
                 rng.uniform(1.38, 1.6), 0.]
        data = _render(100 + i, (s, s), truth)
        start = list(truth)
        start[2] += 15.
        start[3] *= 1.05
        start[4] += 0.03
        holos.append(Hologram(data.reshape(s, s)))
        starts.append(start)
        oracle.append(ofit.fit(data, ofield.meshgrid((s, s)),
                               dict(zip(KEYS, start)),
                               ofield.DEFAULT_INSTRUMENT))
    opt = make_optimizer(starts[0], (8, 8))
    df = opt.optimize_batch(holos, starts=np.array(starts))
    assert len(df) == 16
    for i in range(16):
        o = oracle[i]
        if not o['success']:
            continue
        assert df['success'][i], i
        for k in ('x_p', 'y_p', 'z_p', 'a_p', 'n_p'):
            assert abs(df[k][i] - o[k]) <= TOL[k], (i, k, df[k][i], o[k])


def test_fit_edge_cases():
    from pylorenzmie_b200 import Hologram
    opt = make_optimizer([4., 4., 150., 0.75, 1.45, 0.], (8, 8))
    # empty batch
    df = opt.optimize_batch([], starts=np.zeros((0, 6)))
    assert len(df) == 0
    # fewer pixels than variables: MINPACK's improper input
    tiny = Hologram(np.ones((2, 2)))
    with pytest.raises(ValueError):
        opt.optimize(tiny)
    # non-finite residuals at the start point
    bad = np.ones((16, 16))
    bad[3, 3] = np.nan
    with pytest.raises(ValueError):
        opt.optimize(Hologram(bad))
    # in a batch both are reported per feature, the good one still fits
    good = _render(3, (41, 41), [20., 20., 200., 0.75, 1.45, 0.])
    df = opt.optimize_batch(
        [tiny, Hologram(bad), Hologram(good.reshape(41, 41))],
        starts=np.array([[1., 1., 150., .75, 1.45, 0.],
                         [8., 8., 150., .75, 1.45, 0.],
                         [20., 20., 210., .78, 1.47, 0.]]))
    assert list(df['status'][:2]) == [-1, -2]
    assert not df['success'][0] and not df['success'][1]
    assert df['success'][2]
    assert abs(df['a_p'][2] - 0.75) < 0.02


def test_evaluation_cap():
    '''max_nfev reached: every feature stops there with scipy's status 0
    (not a success) and finite statistics, however many rounds the host
    loop has queued ahead; the first evaluation's point is the start.'''
    from pylorenzmie_b200 import Hologram, workloads
    truth, start = workloads.batch_201(12, seed=17)
    opt = make_optimizer(start[0], (201, 201))
    holos = [Hologram(_render(40 + i, (201, 201), truth[i]).reshape(201, 201))
             for i in range(12)]
    full = opt.optimize_batch(holos, starts=start)
    assert (full['nfev'] > 2).all()
    for cap in (1, 2):
        opt.settings = dict(opt.settings, max_nfev=cap)
        df = opt.optimize_batch(holos, starts=start)
        assert (df['nfev'] == cap).all() and (df['status'] == 0).all()
        assert not df['success'].any()
        assert np.isfinite(df['redchi']).all()
        if cap == 1:
            for j, k in enumerate(KEYS[:5]):
                np.testing.assert_array_equal(df[k].to_numpy(), start[:, j])


def test_autotuned_batch_matches_default(tmp_path, monkeypatch):
    from pylorenzmie_b200 import Hologram, workloads, autotune
    monkeypatch.setenv('LMB200_AUTOTUNE_CACHE', str(tmp_path / 'tune.json'))
    autotune._memory.clear()
    truth, start = workloads.batch_201(8, seed=4)
    truth[:, :2] -= 60.  # centre the spheres on 81x81 crops
    start[:, :2] -= 60.
    data = workloads.render(truth, (81, 81), seed=4).cpu().numpy()
    holos = [Hologram(d.astype(float)) for d in data]
    opt = make_optimizer(start[0], (8, 8))
    d0 = opt.optimize_batch(holos, starts=start, autotune=False)
    d1 = opt.optimize_batch(holos, starts=start, autotune=True)
    assert (tmp_path / 'tune.json').exists()
    for k in ('x_p', 'y_p', 'z_p', 'a_p', 'n_p'):
        assert np.all(np.abs(d0[k] - d1[k]) <= TOL[k] * 0.1)


def test_every_launch_shape_gives_the_same_fit():
    '''All evaluation kernels (CTA tiles, warp tiles, packed two-pixel loop)
    on one batch of mixed crops, odd tile ends and explicit-coordinate
    features included: the same fit as shape 0.  The shapes sum the normal
    equations in different orders, so on small crops, where the chi^2
    surface is flat within FP32 rounding, the stopping point may move: each
    parameter must agree within the target or a third of its uncertainty,
    and chi^2 to 1e-3.'''
    import torch
    from pylorenzmie_b200 import autotune, Instrument, _native
    from pylorenzmie_b200.analysis import _fit
    rng = np.random.default_rng(11)
    items, starts = [], []
    for i in range(12):
        s = int(rng.choice([61, 71, 81, 101]))
        c = (s - 1) / 2.
        truth = [c + rng.uniform(-2, 2), c + rng.uniform(-2, 2),
                 rng.uniform(120., 200.), rng.uniform(0.8, 1.2),
                 rng.uniform(1.38, 1.6), 0.]
        data = _render(500 + i, (s, s), truth)
        start = list(truth)
        start[2] += 12.
        start[3] *= 1.04
        start[4] += 0.02
        if i % 3 == 2:  # a random 60 % of the pixels, explicit coordinates
            keep = rng.random(s * s) < 0.6
            coords = ofield.meshgrid((s, s))[:, keep]
            items.append((data[keep], None, coords))
        else:
            items.append((data, (0., 0., s, s), None))
        starts.append(start)
    starts = np.array(starts)
    inst = Instrument()
    variables = ['x_p', 'y_p', 'z_p', 'a_p', 'n_p']
    packed = _fit.PackedFeatures(items)
    ref = None
    for idx, tpb, ppt, minb in autotune.shapes():
        d_feat, d_data, d_coords, d_params = _fit.upload(packed, starts)
        d_res, _ = _fit.fit_device(d_feat, d_data, d_coords, d_params, 12,
                                   packed.total, inst, variables, None,
                                   None, starts, tile_config=idx)
        p = d_params.view(torch.float64).reshape(12, 6).cpu().numpy()
        r = d_res[:12 * _native.RESULT_DTYPE.itemsize].cpu().numpy().view(
            _native.RESULT_DTYPE)
        assert r['success'].all(), idx
        if ref is None:
            ref, rref = p, r.copy()
            continue
        for j, k in enumerate(KEYS[:5]):
            bound = np.maximum(TOL[k], rref['dparams'][:, j] / 3.)
            assert np.all(np.abs(p[:, j] - ref[:, j]) <= bound), \
                (idx, tpb, ppt, minb, k, p[:, j] - ref[:, j], bound)
        assert np.all(np.abs(r['redchi'] / rref['redchi'] - 1) < 1e-3), idx


def test_streamed_batch_is_bit_identical():
    '''optimize_batch streamed in portions (the fit starts on the first
    features while the rest are converted and copied) gives exactly the
    per-feature results of the one-shot call: a feature's sums do not
    depend on the other features in its batch or on when it was admitted.'''
    from pylorenzmie_b200 import Hologram, workloads
    truth, start = workloads.batch_201(24, seed=9)
    truth[:, :2] -= 60.
    start[:, :2] -= 60.
    data = workloads.render(truth, (81, 81), seed=9).cpu().numpy()
    holos = [Hologram(d.astype(float)) for d in data]
    opt = make_optimizer(start[0], (8, 8))
    d1 = opt.optimize_batch(holos, starts=start, autotune=False, chunks=1)
    for chunks in (3, 24):
        d3 = opt.optimize_batch(holos, starts=start, autotune=False,
                                chunks=chunks)
        assert len(d3) == 24 and list(d3.columns) == list(d1.columns)
        for col in d1.columns:
            np.testing.assert_array_equal(d1[col].to_numpy(),
                                          d3[col].to_numpy())


def test_streamed_fit_withdraw_and_timeout():
    '''lmb_fit_batch_streamed: features admitted before a withdrawal are
    fitted, the rest end with status -4; with nothing admitted the call
    gives up after wait_seconds with LMB_ERR_TIMEOUT (host-side limit, no
    kernel waits).'''
    import torch
    from pylorenzmie_b200 import Instrument, _native
    from pylorenzmie_b200.analysis import _fit
    truth = np.array([[20.3, 19.6, 150., 0.75, 1.45, 0.]] * 6)
    items = [(_render(40 + i, (41, 41), truth[i]), (0., 0., 41, 41), None)
             for i in range(6)]
    starts = truth.copy()
    starts[:, 2] += 8.
    packed = _fit.PackedFeatures(items)
    inst = Instrument()
    variables = ['x_p', 'y_p', 'z_p', 'a_p', 'n_p']
    d_feat, d_data, d_coords, d_params = _fit.upload(packed, starts)
    ready = torch.tensor([-1], dtype=torch.int32, device=d_data.device)
    # withdrawn before anything was admitted
    d_res, _ = _fit.fit_device(d_feat, d_data, d_coords, d_params, 6,
                               packed.total, inst, variables, None, None,
                               starts, ready=ready, wait_seconds=5.)
    r = d_res.cpu().numpy().view(_native.RESULT_DTYPE)
    assert list(r['status']) == [-4] * 6 and not r['success'].any()
    # three admitted, then the producer stops without withdrawing
    d_feat, d_data, d_coords, d_params = _fit.upload(packed, starts)
    ready.fill_(3)
    with pytest.raises(_native.LMBError) as e:
        _fit.fit_device(d_feat, d_data, d_coords, d_params, 6, packed.total,
                        inst, variables, None, None, starts, ready=ready,
                        wait_seconds=0.5)
    assert e.value.status == _native.LMB_ERR_TIMEOUT


def test_distributed_fit_single_rank_is_optimize_batch():
    '''optimize_batch_distributed without a process group (one rank) is
    optimize_batch, rows in input order.'''
    from pylorenzmie_b200 import Hologram, workloads
    from pylorenzmie_b200.distributed import optimize_batch_distributed
    truth, start = workloads.batch_201(6, seed=21)
    truth[:, :2] -= 70.
    start[:, :2] -= 70.
    data = workloads.render(truth, (61, 61), seed=21).cpu().numpy()
    holos = [Hologram(d.astype(float)) for d in data]
    opt = make_optimizer(start[0], (8, 8))
    d0 = opt.optimize_batch(holos, starts=start, autotune=False)
    d1 = optimize_batch_distributed(opt, holos, starts=start, autotune=False)
    for col in d0.columns:
        np.testing.assert_array_equal(d0[col].to_numpy(), d1[col].to_numpy())


def test_stream_matches_batch():
    '''optimize_stream (pipelined batches: conversion and copy of one
    batch overlap the fit of the previous) yields, batch by batch, exactly
    what optimize_batch returns; an empty batch in the stream gives an
    empty frame.'''
    from pylorenzmie_b200 import Hologram, workloads
    batches = []
    for seed in range(4):
        truth, start = workloads.batch_201(6 + seed, seed=30 + seed)
        truth[:, :2] -= 60.
        start[:, :2] -= 60.
        data = workloads.render(truth, (81, 81), seed=30 + seed).cpu().numpy()
        batches.append(([Hologram(d.astype(float)) for d in data], start))
    batches.insert(2, ([], np.zeros((0, 6))))
    opt = make_optimizer(batches[0][1][0], (8, 8))
    ref = [opt.optimize_batch(h, starts=s, autotune=False, chunks=1)
           for h, s in batches]
    got = list(opt.optimize_stream(iter(batches), autotune=False))
    assert len(got) == len(ref)
    for a, b in zip(ref, got):
        assert len(a) == len(b)
        for col in a.columns:
            np.testing.assert_array_equal(a[col].to_numpy(), b[col].to_numpy())
