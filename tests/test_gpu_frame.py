'''GPU: full-frame holograms (1280x1024, 1-16 spheres) and batched fits of
larger mixed crops, against the FP64 oracle.

Frames: the FP32 kernel against the FP64 kernel on every pixel, and against
the numpy oracle on 20 000 random pixels of the frame plus its brightest
pixels (the oracle over the whole frame would take minutes).  Tolerance per
pixel: 2e-5 absolute.  Big spheres close to the focal plane focus light to
H of 20-70 on their axis, where FP32 sums are off by up to ~1e-4; the FP32
kernel bounds its own error per pixel and those pixels are summed again in
FP64 (lmb_hologram), so no pixel may exceed 2e-5.
'''
import numpy as np
import pytest

from oracle import field as ofield, fit as ofit

pytestmark = pytest.mark.gpu

KEYS = ('x_p', 'y_p', 'z_p', 'a_p', 'n_p', 'k_p')


def bench_frame():
    '''The 16-sphere frame that bench.py times.'''
    from pylorenzmie_b200 import workloads
    return workloads.bench_frame()


@pytest.mark.parametrize('seed', [0, 1, 2, 'bench'])
def test_frame_fp32_vs_fp64_and_oracle(seed):
    from pylorenzmie_b200 import LorenzMie, workloads
    P = bench_frame() if seed == 'bench' else workloads.frame(seed=seed)
    spheres = workloads.spheres(P)
    coords = LorenzMie.meshgrid((1024, 1280))
    h32 = LorenzMie(coordinates=coords, particle=spheres).hologram()
    h64 = LorenzMie(coordinates=coords, particle=spheres,
                    double_precision=True).hologram()
    assert h32.shape == (1024 * 1280,)
    assert np.all(np.abs(h32 - h64) <= 2e-5)
    rng = np.random.default_rng(7 if seed == 'bench' else seed)
    idx = rng.choice(coords.shape[1], 20000, replace=False)
    # and the brightest pixels, where FP32 alone would miss the tolerance
    idx = np.union1d(idx, np.argsort(h64)[-200:])
    sub = coords[:, idx]
    ref = ofield.hologram(sub, [dict(zip(KEYS, p)) for p in P],
                          ofield.DEFAULT_INSTRUMENT)
    assert np.abs(h64[idx] - ref).max() <= 1e-10
    assert np.all(np.abs(h32[idx] - ref) <= 2e-5)
    # the same pixels as an explicit coordinate list give the same values
    m = LorenzMie(coordinates=sub, particle=spheres)
    assert np.abs(m.hologram() - h32[idx]).max() <= 1e-6


def test_frames_fp32_within_2e5_many_seeds():
    '''Every pixel of 20 more seeded frames (1-16 spheres each) within
    2e-5 of the FP64 kernel, which is itself pinned to the oracle above.'''
    import torch
    from pylorenzmie_b200 import LorenzMie, workloads
    coords = LorenzMie.meshgrid((1024, 1280))
    m32 = LorenzMie(coordinates=coords)
    m64 = LorenzMie(coordinates=coords, double_precision=True)
    worst = 0.
    for seed in range(3, 23):
        spheres = workloads.spheres(workloads.frame(seed=seed))
        m32.particle = spheres
        m64.particle = spheres
        d = (m32.hologram(device=True).double() -
             m64.hologram(device=True)).abs().max().item()
        worst = max(worst, d)
        assert d <= 2e-5, (seed, d)
    assert worst > 0.


def test_frame_batch_items_fp64_resum():
    '''Several frames in one launch (batch_hologram): each item's marked
    pixels are summed again in FP64.'''
    from pylorenzmie_b200 import LorenzMie, workloads
    coords = LorenzMie.meshgrid((256, 320))
    lists, refs = [], []
    for seed in range(3):
        P = workloads.frame(seed=seed, shape=(256, 320))[:4]
        P[0] = [160.3, 127.8, 2.9 / 0.048 + 10., 2.9, 1.55, 0.]
        lists.append(workloads.spheres(P))
        refs.append(LorenzMie(coordinates=coords, particle=lists[-1],
                              double_precision=True).hologram())
    m = LorenzMie(coordinates=coords)
    h = m.batch_hologram(lists)
    for i in range(3):
        assert np.abs(h[i] - refs[i]).max() <= 2e-5
        assert refs[i].max() > 20.


def test_fit_mixed_large_crops_vs_oracle():
    from pylorenzmie_b200 import LorenzMie, Optimizer, Hologram, workloads
    sides = np.array([151, 201, 251, 301])
    rng = np.random.default_rng(5)
    truth = np.zeros((4, 6))
    c = (sides - 1) / 2.
    truth[:, 0] = c + rng.uniform(-2, 2, 4)
    truth[:, 1] = c + rng.uniform(-2, 2, 4)
    truth[:, 2] = [180., 200., 220., 240.]
    truth[:, 3] = [0.6, 0.75, 0.9, 1.1]
    truth[:, 4] = [1.40, 1.42, 1.45, 1.50]
    start = truth.copy()
    start[:, 3] *= 1.05
    start[:, 4] += 0.03
    start[:, 2] += 15.
    holos, oracle = [], []
    for i, s in enumerate(sides):
        g = ofield.meshgrid((s, s))
        h = ofield.hologram(g, [dict(zip(KEYS, truth[i]))],
                            ofield.DEFAULT_INSTRUMENT)
        d = h + np.random.default_rng(40 + i).normal(0., 0.05, h.shape)
        holos.append(Hologram(d.reshape(s, s)))
        oracle.append(ofit.fit(d, g, dict(zip(KEYS, start[i])),
                               ofield.DEFAULT_INSTRUMENT))
    opt = Optimizer(model=LorenzMie(coordinates=np.zeros((2, 1))))
    df = opt.optimize_batch(holos, starts=start)
    tol = {'x_p': 0.02, 'y_p': 0.02, 'z_p': 0.02, 'a_p': 1e-3, 'n_p': 1e-4}
    for i in range(4):
        assert df['success'][i] and oracle[i]['success']
        assert df['npix'][i] == sides[i] ** 2
        for k, t in tol.items():
            assert abs(df[k][i] - oracle[i][k]) <= t, (i, k)
        assert abs(df['redchi'][i] / oracle[i]['redchi'] - 1) < 1e-3


@pytest.mark.parametrize('spheres_um', [(12.,), (6., 9.), (24.,)])
def test_large_spheres_resum_per_thread(spheres_um):
    '''One or two large spheres (n_max 120-490): their error bound marks
    most pixels, and with so few particles the FP64 re-sum takes one thread
    per marked pixel rather than one lane per particle.  Every pixel stays
    within 2e-5 of the FP64 kernel, and the FP64 kernel matches the oracle
    on sampled pixels.'''
    from pylorenzmie_b200 import LorenzMie, workloads
    shape = (384, 448)
    P = np.zeros((len(spheres_um), 6))
    for i, a in enumerate(spheres_um):
        P[i] = [130. + 180. * i, 190. - 20. * i, a / 0.048 + 40., a, 1.45, 0.]
    spheres = workloads.spheres(P)
    coords = LorenzMie.meshgrid(shape)
    h32 = LorenzMie(coordinates=coords, particle=spheres).hologram()
    h64 = LorenzMie(coordinates=coords, particle=spheres,
                    double_precision=True).hologram()
    assert np.all(np.abs(h32 - h64) <= 2e-5)
    rng = np.random.default_rng(3)
    idx = np.union1d(rng.choice(coords.shape[1], 400, replace=False),
                     np.argsort(h64)[-20:])
    ref = ofield.hologram(coords[:, idx], [dict(zip(KEYS, p)) for p in P],
                          ofield.DEFAULT_INSTRUMENT)
    assert np.abs(h64[idx] - ref).max() <= 1e-9
