'''Host-side behaviour of the drop-in classes, mirroring the reference's
structural tests (tests/test_lorenzmie.py, test_sphere.py, test_optimizer.py,
test_hologram.py, test_mask.py) -- no GPU needed.'''
import json

import numpy as np
import pandas as pd
import pytest

from pylorenzmie_b200 import (LorenzMie, Sphere, Instrument, Particle,
                              Optimizer, Hologram, Mask, meshgrid, workloads)
from pylorenzmie_b200.analysis import _fit
from pylorenzmie_b200 import _native


def test_meshgrid():
    xy = meshgrid((32, 24), flatten=False)
    assert xy.shape == (2, 32, 24)
    xy = meshgrid((32, 24))
    assert xy.shape == (2, 32 * 24)
    assert xy[0, 1] == 1 and xy[1, 24] == 1
    c = meshgrid((2, 3), corner=(10., 5.))
    assert c[0, 0] == 10. and c[1, 0] == 5.


def test_model_coordinates():
    m = LorenzMie()
    assert m.coordinates.shape == (3, 201 * 201)
    assert m.method == 'b200 numpy' and 'numpy' in m.method
    point = np.array([1, 2, 3]).reshape((3, 1))
    m.coordinates = point
    assert np.allclose(m.coordinates, point)
    m.coordinates = np.arange(256)
    assert m.coordinates.shape[0] == 3
    c = [[1, 1, 1, 1], [2, 2, 2, 2], [3, 3, 3, 3]]
    m.coordinates = c
    assert np.allclose(m.coordinates, np.array(c))
    with pytest.raises(ValueError):
        m.coordinates = np.zeros((4, 5))


def test_model_properties_and_json():
    m = LorenzMie()
    m.properties = dict(x_p=-42)
    assert m.particle.x_p == -42
    m.properties = dict(n_m=1.5, noise=0.1)
    assert m.instrument.n_m == 1.5 and m.instrument.noise == 0.1
    keys = list(m.properties)
    assert keys[:6] == ['x_p', 'y_p', 'z_p', 'a_p', 'n_p', 'k_p']
    assert keys[6:] == ['n_m', 'wavelength', 'magnification',
                        'numerical_aperture', 'noise']
    m.particle.n_p = 1.5
    s = m.to_json()
    m.particle.n_p = 1.4
    m.from_json(s)
    assert m.particle.n_p == 1.5
    assert isinstance(m.to_pandas(), pd.Series)
    assert 'LorenzMie' in repr(m)
    assert m.jac_params == frozenset(('x_p', 'y_p', 'z_p', 'a_p', 'n_p',
                                      'k_p'))


def test_sphere_and_instrument():
    s = Sphere()
    assert (s.a_p, s.n_p, s.k_p) == (1., 1.5, 0.)
    s.d_p = 3.
    assert s.a_p == 1.5 and s.d_p == 3.
    for key in ('x_p', 'y_p', 'z_p', 'a_p', 'n_p', 'k_p'):
        assert key in s.properties
    props = s.properties
    props['a_p'] += 0.25
    s.properties = props
    assert s.a_p == props['a_p']
    assert Sphere.wiscombe_yang(1., 10. + 0.j) == 10
    assert Sphere.wiscombe_yang(10., 10. + 0.j) == 100
    assert Sphere.wiscombe_yang(4210., 10. + 0.j) == 42100
    assert Sphere.neves_pisignano(10.) == 11
    p = Particle()
    assert len(p) == 1 and list(p) == [p] and p[0] is p
    with pytest.raises(IndexError):
        p[1]
    i = Instrument()
    assert abs(i.wavenumber() - 2 * np.pi / 0.447 * 1.34 * 0.048) < 1e-12
    assert abs(i.wavenumber(scaled=False) - 2 * np.pi / 0.447 * 1.34) < 1e-12
    assert abs(i.wavenumber(in_medium=False, scaled=False) -
               2 * np.pi / 0.447) < 1e-12


def test_compute_without_gpu_raises():
    import torch
    if torch.cuda.is_available():
        pytest.skip('a GPU is present')
    m = LorenzMie()
    with pytest.raises(RuntimeError):
        m.hologram()


def test_hologram_container():
    data = np.arange(12.).reshape(3, 4)
    h = Hologram(data, corner=(10., 20.))
    assert h.shape == (3, 4)
    assert h.flat_data.shape == (12,)
    assert h.flat_coordinates.shape == (2, 12)
    assert h.flat_coordinates[0, 0] == 10. and h.flat_coordinates[1, 0] == 20.
    crop = h[1:3, 1:4]
    assert crop.shape == (2, 3) and crop.corner == (11., 21.)
    assert crop.is_grid
    sub = h[::2, ::2]
    assert not sub.is_grid
    assert h == Hologram(data.copy(), corner=(10., 20.))


def test_mask():
    np.random.seed(0)
    m = Mask(shape=(201, 201), fraction=0.2)
    assert abs(m().mean() - 0.2) < 0.01
    excl = np.zeros((201, 201), bool)
    excl[:10] = True
    m.exclude = excl
    assert not m()[:10].any()
    h = Hologram(np.random.rand(50, 40))
    d, c = Mask(fraction=0.3).apply(h)
    assert d.shape[0] == c.shape[1] and c.shape[0] == 2
    assert Mask().properties == {'fraction': 0.1}


@pytest.mark.parametrize('shape,fraction', [((121, 121), 0.1),
                                            ((37, 53), 0.5), ((1, 1), 0.3),
                                            ((0, 5), 0.1), ((64, 64), 1.)])
@pytest.mark.parametrize('excluded', [False, True])
def test_mask_draws_are_numpys(shape, fraction, excluded):
    '''The subset drawn by the library on the global generator is
    np.random.rand(*shape) < fraction with the excluded pixels removed,
    and the generator ends where numpy's own draws leave it.'''
    from pylorenzmie_b200.analysis import Mask, Hologram
    exclude = None
    if excluded:
        exclude = np.random.default_rng(1).random(shape) < 0.3
    np.random.seed(7)
    state = np.random.get_state()
    m = Mask(fraction=fraction, exclude=exclude)
    m.shape = shape
    after = np.random.rand(3)
    np.random.set_state(state)
    ref = np.random.rand(*shape) < fraction
    if exclude is not None:
        ref[exclude] = False
    assert np.array_equal(m(), ref)
    assert np.array_equal(np.random.rand(3), after)
    if 0 not in shape:
        h = Hologram(np.random.default_rng(2).random(shape),
                     corner=(3., 5.))
        np.random.set_state(state)
        data, coords = m.apply(h)
        np.random.set_state(state)
        want = np.random.rand(*shape) < fraction
        if exclude is not None:
            want[exclude] = False
        assert np.array_equal(data, h.data[want])
        assert np.array_equal(coords, h.coordinates[:, want])


def test_mask_mt19937_layouts_agree():
    '''lmb_mask_select's two layouts -- through next_double, and numpy's
    MT19937 words advanced a block at a time -- give the same subsets and
    leave the generator in the same state, for draws that straddle blocks
    (a double takes two of a block's 624 words).'''
    import ctypes
    import importlib
    mask_module = importlib.import_module('pylorenzmie_b200.analysis.Mask')
    assert mask_module._mt_blocks_ok()
    lib = _native.load()
    g = [np.random.MT19937(99), np.random.MT19937(99)]
    for n, frac in [(0, 0.1), (1, 0.9), (311, 0.1), (312, 0.5), (313, 0.5),
                    (14641, 0.1), (7, 1.0), (5, 0.0)]:
        out = []
        for layout, bg in enumerate(g):
            idx = np.empty(max(n, 1), dtype=np.int64)
            cnt = ctypes.c_longlong()
            assert lib.lmb_mask_select(bg.ctypes.bit_generator.value, n,
                                       frac, None, layout, idx.ctypes.data,
                                       ctypes.byref(cnt)) == _native.LMB_OK
            out.append(idx[:cnt.value].copy())
        assert np.array_equal(out[0], out[1]), n
        s0, s1 = (bg.state['state'] for bg in g)
        assert np.array_equal(s0['key'], s1['key']) and s0['pos'] == s1['pos']


def test_optimizer_configuration():
    opt = Optimizer(model=LorenzMie())
    assert opt.result is None and opt.mask is None
    assert opt.variables == ['x_p', 'y_p', 'z_p', 'a_p', 'n_p']
    for f in ('noise', 'numerical_aperture', 'k_p'):
        assert f in opt.fixed
    opt.variables = ['x_p', 'y_p', 'z_p', 'a_p']
    assert 'n_p' in opt.fixed
    opt.fixed = list(opt.model.properties)[:2]
    assert 'x_p' not in opt.variables
    fixed = ['wavelength']
    o2 = Optimizer(model=opt.model, fixed=fixed)
    fixed.append('n_m')
    assert 'n_m' not in o2.fixed
    opt.robust = True
    assert opt.robust and opt.settings['method'] == 'trf'
    opt.robust = False
    assert opt.settings['method'] == 'lm'
    assert isinstance(opt.metadata, pd.Series)
    props = opt.properties
    opt.properties = props
    assert 'settings' in props
    with pytest.raises(RuntimeError):
        opt.report()
    opt.fraction = 0.25
    assert isinstance(opt.mask, Mask) and opt.fraction == 0.25


def test_optimizer_rejects_incompatible_model():
    class Other:
        method = 'cupy'
    with pytest.raises(TypeError):
        Optimizer(model=Other())


def test_device_fit_selection():
    opt = Optimizer(model=LorenzMie())
    assert opt._device_fit_ok()
    opt.variables = ['x_p', 'y_p', 'z_p', 'a_p', 'n_p', 'k_p']
    assert opt._device_fit_ok()
    opt.variables = ['x_p', 'n_m']
    assert not opt._device_fit_ok()          # instrument parameter free
    opt = Optimizer(model=LorenzMie(), robust=True)
    assert not opt._device_fit_ok()          # trf + cauchy: host loop
    opt = Optimizer(model=LorenzMie())
    opt.model.particle = [Sphere(), Sphere()]
    assert not opt._device_fit_ok()


def test_small_batch_shape():
    '''Batches below SMALL_BATCH features evaluate with one pixel pair a
    thread (256 threads x 2 pixels); larger ones keep the default shape.'''
    import ctypes
    lib = _native.load()
    tpb, ppt, minb = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    assert lib.lmb_fit_tile_config(_fit.SMALL_SHAPE, ctypes.byref(tpb),
                                   ctypes.byref(ppt), ctypes.byref(minb)) == 0
    assert (tpb.value, ppt.value) == (256, 2)
    assert _fit.default_shape(1) == _fit.default_shape(63) == _fit.SMALL_SHAPE
    assert _fit.default_shape(64) == _fit.default_shape(256) == 0


def test_packed_features_layout():
    a = np.ones((3, 4))
    b = np.arange(6.)
    items = [(a, (1., 2., 3, 4), None),
             (b, None, np.vstack([np.arange(6.), np.zeros(6)]))]
    p = _fit.PackedFeatures(items)
    f = p.features
    assert f.dtype == _native.FEATURE_DTYPE
    assert list(f['npix']) == [12, 6] and list(f['data_offset']) == [0, 12]
    assert (f['nx'][0], f['ny'][0], f['x0'][0], f['y0'][0]) == (4, 3, 1., 2.)
    assert f['nx'][1] == 0
    assert p.data.dtype == np.float32 and p.data.size == 18
    xy = p.coords.reshape(-1, 2)
    assert xy.shape == (18, 2)
    assert tuple(xy[1]) == (2., 2.) and tuple(xy[4]) == (1., 3.)
    assert tuple(xy[12 + 5]) == (5., 0.)
    with pytest.raises(ValueError):
        _fit.PackedFeatures([(np.ones(5), (0., 0., 2, 2), None)])
    assert _fit.variable_mask(['x_p', 'k_p']) == 0b100001


def test_fit_capacity_covers_growth():
    starts = np.array([[0, 0, 200, 0.75, 1.42, 0.]])
    cap = _fit.fit_capacity(starts, 1.34, 0.447)
    nm = Sphere.wiscombe_yang(2 * np.pi / 0.447 * 1.34 * 0.75 * 1.25,
                              (1.42 + 0.25) / 1.34)
    assert cap >= nm


def test_workloads():
    truth, start = workloads.batch_201(8, seed=1)
    assert truth.shape == (8, 6)
    assert np.all(np.abs(truth[:, :2] - 100) <= 2)
    assert np.allclose(start[:, 3], truth[:, 3] * 1.05)
    sides, t, s = workloads.mixed_crops(64, seed=2)
    assert np.all(sides % 2 == 1) and sides.min() >= 51 and sides.max() <= 301
    p = workloads.frame(seed=3)
    assert 1 <= p.shape[0] <= 16
    assert np.all(p[:, 2] >= p[:, 3] / 0.048 + 10 - 1e-9)
    assert len(workloads.spheres(p)) == p.shape[0]


def test_autotune_keys_and_cache(tmp_path, monkeypatch):
    from pylorenzmie_b200 import autotune
    monkeypatch.setenv('LMB200_AUTOTUNE_CACHE', str(tmp_path / 'tune.json'))
    k1 = autotune.problem_key('B200', 30, 201 * 201)
    k2 = autotune.problem_key('B200', 32, 150 * 150)
    k3 = autotune.problem_key('B200', 33, 201 * 201)
    assert k1 == k2 and k1 != k3
    assert 'layered' in autotune.problem_key('B200', 30, 100, layered=True)
    # batches of up to 64, up to 256 and more are tuned apart
    kb = [autotune.problem_key('B200', 30, 201 * 201, batch=b)
          for b in (32, 64, 65, 256, 257, 1024)]
    assert kb[0] == kb[1] != kb[2] == kb[3] != kb[4] == kb[5]
    assert autotune.cache_path() == tmp_path / 'tune.json'
    autotune._store('x', {'config': 3})
    autotune._memory.clear()
    assert autotune.lookup('x') == {'config': 3}
    assert autotune.lookup('missing') is None
    shapes = autotune.shapes()
    assert len(shapes) >= 2 and shapes[0][0] == 0
    assert all(t % 32 == 0 and 512 % p == 0 for _, t, p, _ in shapes)


def test_pipeline_chunking():
    from pylorenzmie_b200.analysis import _fit
    npix = np.array([201 * 201] * 256)
    assert _fit.default_chunks(npix) == 8
    assert _fit.default_chunks(npix[:4]) == 1
    assert _fit.default_chunks(np.array([2500] * 64)) == 1
    rng = np.random.default_rng(0)
    for n, c in [(10, 3), (256, 4), (5, 4), (1, 2)]:
        px = rng.integers(100, 90000, n)
        r = _fit.split_by_pixels(px, c)
        assert r[0][0] == 0 and r[-1][1] == n
        assert all(a < b for a, b in r)
        assert all(r[i][1] == r[i + 1][0] for i in range(len(r) - 1))
        assert len(r) <= c
    r = _fit.split_by_pixels(np.full(100, 7), 4)
    assert [b - a for a, b in r] == [25, 25, 25, 25]


def test_packed_write_range_any_cut():
    '''write_range converts exactly the crops asked for, whatever the crop
    sizes and the thread cuts (cuts fall inside crops).'''
    from pylorenzmie_b200.analysis import _fit
    rng = np.random.default_rng(3)
    items = []
    for i in range(37):
        n = int(rng.integers(1, 90000))
        items.append((rng.random(n), None, np.zeros((2, n))))
    pk = _fit.PackedFeatures(items)
    ref = np.concatenate([it[0] for it in items]).astype(np.float32)
    out = np.full(pk.total, -1., np.float32)
    pk.write_range(out, 5, 23)
    a = pk.features['data_offset'][5]
    b = pk.features['data_offset'][22] + pk.features['npix'][22]
    np.testing.assert_array_equal(out[a:b], ref[a:b])
    assert np.all(out[:a] == -1.) and np.all(out[b:] == -1.)
    np.testing.assert_array_equal(pk.write_data(np.empty(pk.total, np.float32)),
                                  ref)


def test_chi2_workspace_blocks_of_128():
    '''The population chi^2 partials: one per 128-pixel block of the largest
    crop and per item (a DE crop of 293 pixels takes 3 blocks), then an
    int flag per partial; 0 for an empty launch.'''
    lib = _native.load()
    for npts, nitems in [(293, 960), (128, 1), (129, 7), (40401, 3)]:
        nb = (npts + 127) // 128
        n = nb * nitems
        want = (n * 8 + 255) // 256 * 256 + n * 4
        assert lib.lmb_chi2_workspace_bytes(npts, nitems) == want
    assert lib.lmb_chi2_workspace_bytes(0, 5) == 0
    assert lib.lmb_chi2_workspace_bytes(10, 0) == 0
