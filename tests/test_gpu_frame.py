'''GPU: full-frame holograms (1280x1024, 1-16 spheres) and batched fits of
larger mixed crops, against the FP64 oracle.

Frames: the FP32 kernel against the FP64 kernel on every pixel, and against
the numpy oracle on 20 000 random pixels of the frame (the oracle over the
whole frame would take minutes).  Tolerance per pixel: 2e-5 + 2e-6 H.  Big
spheres close to the focal plane focus light to H of 20-60 on the axis,
where FP32 rounding of the order coefficients alone (about 6 ulp of the
field) exceeds 2e-5 absolute; the relative error stays below 2e-6.
'''
import numpy as np
import pytest

from oracle import field as ofield, fit as ofit

pytestmark = pytest.mark.gpu

KEYS = ('x_p', 'y_p', 'z_p', 'a_p', 'n_p', 'k_p')


@pytest.mark.parametrize('seed', [0, 1, 2])
def test_frame_fp32_vs_fp64_and_oracle(seed):
    from pylorenzmie_b200 import LorenzMie, workloads
    P = workloads.frame(seed=seed)
    spheres = workloads.spheres(P)
    coords = LorenzMie.meshgrid((1024, 1280))
    h32 = LorenzMie(coordinates=coords, particle=spheres).hologram()
    h64 = LorenzMie(coordinates=coords, particle=spheres,
                    double_precision=True).hologram()
    assert h32.shape == (1024 * 1280,)
    assert np.all(np.abs(h32 - h64) <= 2e-5 + 2e-6 * h64)
    rng = np.random.default_rng(seed)
    idx = rng.choice(coords.shape[1], 20000, replace=False)
    sub = coords[:, idx]
    ref = ofield.hologram(sub, [dict(zip(KEYS, p)) for p in P],
                          ofield.DEFAULT_INSTRUMENT)
    assert np.abs(h64[idx] - ref).max() <= 1e-10
    assert np.all(np.abs(h32[idx] - ref) <= 2e-5 + 2e-6 * ref)
    # the same pixels as an explicit coordinate list give the same values
    m = LorenzMie(coordinates=sub, particle=spheres)
    assert np.abs(m.hologram() - h32[idx]).max() <= 1e-6


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
