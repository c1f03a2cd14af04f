'''Seeded synthetic workloads of the benchmark configurations.

No public dataset is involved: every input is drawn from a seeded
``numpy.random.default_rng`` with the shapes and distributions below, and
holograms are rendered with the FP64 per-pixel kernel plus Gaussian noise
of sigma = 0.05 (the instrument's noise).

* single_201  -- one 201x201 crop: a_p = 0.75 um, n_p = 1.42, k_p = 0,
  x_p, y_p = 100 + U(-2, 2) px, z_p = 200 px; start perturbed by 5 % in
  a_p, +0.02 in n_p and +10 px in z_p.  ``batch_201`` stacks B of them.
* frame       -- a 1280x1024 frame with 1..16 spheres (seeded count),
  a_p ~ U(0.4, 3.0) um, n_p ~ U(1.38, 1.70), k_p ~ U(0, 1e-3),
  z_p ~ U(50, 600) px constrained to z_p >= a_p/magnification + 10 px so
  that the focal plane never cuts through a sphere, positions uniform
  over the frame.
* mixed_crops -- B features of square odd crops of side U{51, 53, .., 301}
  with single_201's parameters centred on the crop; start perturbed by
  5 % in a_p, +0.03 in n_p and +15 px in z_p.
* large       -- crops of 401x401 with a_p ~ U(3, 6) um, n_p ~ U(1.4, 2.0),
  z_p ~ U(200, 600) px.
* layered     -- three-layer core-shell spheres in crops of 101..201 px
  (the video-stream workload; see ``layered``).
* estimate_frame -- a 1280x640 frame of 32 spheres on an 8x4 grid of
  160 px pitch (+-3 px), z_p ~ U(100, 300) px, a_p ~ U(0.5, 1.5) um,
  n_p ~ U(1.38, 1.60), with a 121x121 box around each (the global-estimate
  workload of a frame's features).
'''
import numpy as np

KEYS = ('x_p', 'y_p', 'z_p', 'a_p', 'n_p', 'k_p')
NOISE = 0.05


def batch_201(B, seed=0):
    '''Truth and start parameters (B, 6) for 201x201 crops.'''
    rng = np.random.default_rng(seed)
    truth = np.zeros((B, 6))
    truth[:, 0] = 100. + rng.uniform(-2., 2., B)
    truth[:, 1] = 100. + rng.uniform(-2., 2., B)
    truth[:, 2] = 200.
    truth[:, 3] = 0.75
    truth[:, 4] = 1.42
    start = truth.copy()
    start[:, 3] *= 1.05
    start[:, 4] += 0.02
    start[:, 2] += 10.
    return truth, start


def mixed_crops(B, seed=0):
    '''Crop sides (B,), truth and start (B, 6) for mixed crop sizes.'''
    rng = np.random.default_rng(seed)
    sides = 2 * rng.integers(25, 151, B) + 1          # 51 .. 301, odd
    truth = np.zeros((B, 6))
    c = (sides - 1) / 2.
    truth[:, 0] = c + rng.uniform(-2., 2., B)
    truth[:, 1] = c + rng.uniform(-2., 2., B)
    truth[:, 2] = 200.
    truth[:, 3] = 0.75
    truth[:, 4] = 1.42
    start = truth.copy()
    start[:, 3] *= 1.05
    start[:, 4] += 0.03
    start[:, 2] += 15.
    return sides, truth, start


def frame(seed=0, shape=(1024, 1280), magnification=0.048):
    '''Sphere parameters (n, 6) of one frame.'''
    rng = np.random.default_rng(seed)
    n = int(rng.integers(1, 17))
    p = np.zeros((n, 6))
    p[:, 3] = rng.uniform(0.4, 3.0, n)
    p[:, 4] = rng.uniform(1.38, 1.70, n)
    p[:, 5] = rng.uniform(0., 1e-3, n)
    zmin = p[:, 3] / magnification + 10.
    p[:, 2] = np.maximum(rng.uniform(50., 600., n), zmin)
    p[:, 0] = rng.uniform(0., shape[1], n)
    p[:, 1] = rng.uniform(0., shape[0], n)
    return p


def estimate_frame(n=32, seed=21, instrument=None, device=None):
    '''(params (n, 6), frame (640, 1280) float64 numpy, boxes) of the
    estimate workload: the FP32 hologram of the n spheres plus noise, and
    one ((x0, y0), 121, 121) box per sphere.'''
    from .theory import LorenzMie, Instrument
    inst = instrument or Instrument()
    rng = np.random.default_rng(seed)
    p = np.zeros((n, 6))
    p[:, 0] = 80. + 160. * (np.arange(n) % 8) + rng.uniform(-3., 3., n)
    p[:, 1] = 80. + 160. * (np.arange(n) // 8) + rng.uniform(-3., 3., n)
    p[:, 2] = rng.uniform(100., 300., n)
    p[:, 3] = rng.uniform(0.5, 1.5, n)
    p[:, 4] = rng.uniform(1.38, 1.60, n)
    m = LorenzMie(coordinates=LorenzMie.meshgrid((640, 1280)),
                  particle=spheres(p), instrument=inst, device=device)
    data = (m.hologram() + rng.normal(0., inst.noise, 640 * 1280)
            ).reshape(640, 1280)
    boxes = [((int(x) - 60, int(y) - 60), 121, 121) for x, y in p[:, :2]]
    return p, data, boxes


def large(B, seed=0, side=401):
    rng = np.random.default_rng(seed)
    p = np.zeros((B, 6))
    c = (side - 1) / 2.
    p[:, 0] = c + rng.uniform(-2., 2., B)
    p[:, 1] = c + rng.uniform(-2., 2., B)
    p[:, 2] = rng.uniform(200., 600., B)
    p[:, 3] = rng.uniform(3., 6., B)
    p[:, 4] = rng.uniform(1.4, 2.0, B)
    return p


def layered(B, seed=0, magnification=0.048):
    '''Three-layer core-shell features of the video-stream workload:
    crop sides U{101, 103, .., 201}, radius fractions ~U(0.3, 0.9) nested
    (sorted), layer indices ~U(1.33, 1.80), outer a_p ~U(0.5, 2.5) um,
    z_p ~U(150, 400) px (at least a_p/magnification + 10 px), centred
    +-2 px.  Returns sides (B,), params (B, 6), fractions (B, 2) and inner
    indices (B, 2).  Starts: a_p +5 %, n_p +0.02, z_p +10 px.'''
    rng = np.random.default_rng(seed)
    sides = 2 * rng.integers(50, 101, B) + 1
    frac = np.sort(rng.uniform(0.3, 0.9, (B, 2)), axis=1)
    idx = rng.uniform(1.33, 1.80, (B, 3))
    p = np.zeros((B, 6))
    c = (sides - 1) / 2.
    p[:, 0] = c + rng.uniform(-2., 2., B)
    p[:, 1] = c + rng.uniform(-2., 2., B)
    p[:, 3] = rng.uniform(0.5, 2.5, B)
    p[:, 2] = np.maximum(rng.uniform(150., 400., B),
                         p[:, 3] / magnification + 10.)
    p[:, 4] = idx[:, 2]
    start = p.copy()
    start[:, 3] *= 1.05
    start[:, 4] += 0.02
    start[:, 2] += 10.
    return sides, p, start, frac, idx[:, :2].astype(complex)


def layered_spheres(params, fractions, core_indices):
    from .theory import LayeredSphere
    out = []
    for row, f, c in zip(np.atleast_2d(params), fractions, core_indices):
        s = LayeredSphere(a_p=row[3], n_p=row[4], k_p=row[5],
                          fractions=tuple(f), core_indices=tuple(c))
        s.r_p = row[:3]
        out.append(s)
    return out


def spheres(params):
    '''Sphere objects from a (n, 6) parameter array.'''
    from .theory import Sphere
    out = []
    for row in np.atleast_2d(params):
        s = Sphere(a_p=row[3], n_p=row[4], k_p=row[5])
        s.r_p = row[:3]
        out.append(s)
    return out


def render(params, shape, seed=0, instrument=None, device=None,
           noise=NOISE):
    '''Noisy holograms (B, ny, nx) float32 of one sphere each, rendered by
    the FP64 kernel on the device; same crop shape for the whole batch.'''
    import torch
    from .theory import LorenzMie, Instrument
    inst = instrument or Instrument()
    m = LorenzMie(coordinates=LorenzMie.meshgrid(shape), instrument=inst,
                  double_precision=True, device=device)
    lists = [[s] for s in spheres(params)]
    h = m.batch_hologram(lists, device=True)
    g = torch.Generator(device=h.device)
    g.manual_seed(int(seed))
    h = h + noise * torch.randn(h.shape, generator=g, device=h.device,
                                dtype=h.dtype)
    return h.float().reshape(len(lists), *shape)


def render_particles(particles, shapes, seed=0, instrument=None, device=None,
                     noise=NOISE):
    '''Noisy holograms (list of (ny, nx) float32 numpy arrays), one particle
    (Sphere or LayeredSphere) per crop, crops of differing shapes.'''
    import torch
    from .theory import LorenzMie, Instrument
    inst = instrument or Instrument()
    g = torch.Generator(device='cuda' if device is None else device)
    g.manual_seed(int(seed))
    out = []
    for p, shape in zip(particles, shapes):
        m = LorenzMie(coordinates=LorenzMie.meshgrid(shape), particle=p,
                      instrument=inst, double_precision=True, device=device)
        h = m.hologram(device=True)
        h = h + noise * torch.randn(h.shape, generator=g, device=h.device,
                                    dtype=h.dtype)
        out.append(h.float().reshape(shape).cpu().numpy())
    return out


def _run_estimate_frame(device_search, repeat, optimize=False):
    '''Frame.estimate of the estimate workload, ``repeat`` times (the first
    one warms up), and with ``optimize`` Frame.optimize after each; prints
    the seconds each took.'''
    import time
    import torch
    from .theory import Instrument
    from .analysis import Frame
    inst = Instrument()
    _, data, boxes = estimate_frame(32, 21, inst)
    for rep in range(repeat):
        f = Frame(instrument=inst)
        f.data = data
        f.bboxes = boxes
        for i, feat in enumerate(f.features):
            feat.estimator.seed = 40 + i
            feat.estimator.device_search = device_search
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        f.estimate()
        torch.cuda.synchronize()
        print(f'estimate_frame {rep}: {time.perf_counter() - t0:.4f} s')
        if optimize:
            t0 = time.perf_counter()
            f.optimize()
            torch.cuda.synchronize()
            print(f'optimize_frame {rep}: {time.perf_counter() - t0:.4f} s')


def bench_frame():
    '''Sphere parameters (16, 6) of the frame that bench.py times: seeded
    frames stacked until 16 spheres.'''
    p = frame(seed=5)
    while p.shape[0] < 16:
        p = np.vstack([p, frame(seed=5 + p.shape[0])])[:16]
    return p


def _run_frame(repeat, fp64=False):
    '''LorenzMie.hologram(device=True) of the 16-sphere 1280x1024 frame,
    ``repeat`` times; prints the milliseconds of each.'''
    import time
    import torch
    from .theory import LorenzMie, Instrument
    m = LorenzMie(coordinates=LorenzMie.meshgrid((1024, 1280)),
                  particle=spheres(bench_frame()), instrument=Instrument(),
                  double_precision=fp64)
    for rep in range(repeat):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        m.hologram(device=True)
        torch.cuda.synchronize()
        print(f'frame {rep}: {(time.perf_counter() - t0) * 1e3:.3f} ms')


# 1280x1024 frames of spheres of one size each (radius um, count), at
# z = a_p / 0.048 + 60 px: the bench's frame, then sizes that make the FP64
# re-sum of the FP32 kernel mark few or most pixels
FRAME_SIZES = ((1.0, 16), (3.0, 16), (6.0, 4), (12.0, 2), (24.0, 1),
               (1.0, 64))


def size_frame(a_p, count, shape=(1024, 1280), seed=1):
    '''Sphere parameters (count, 6): radius a_p (um), n_p 1.5, at
    z = a_p / 0.048 + 60 px, uniform over the frame.'''
    rng = np.random.default_rng(seed)
    p = np.zeros((count, 6))
    p[:, 3] = a_p
    p[:, 4] = 1.5
    p[:, 2] = a_p / 0.048 + 60.
    p[:, 0] = rng.uniform(0, shape[1], count)
    p[:, 1] = rng.uniform(0, shape[0], count)
    return p


def _run_frame_sizes(repeat):
    '''Median CUDA-event milliseconds of LorenzMie.hologram(device=True) for
    the bench frame and each FRAME_SIZES frame.'''
    import torch
    from .theory import LorenzMie, Instrument
    from .theory import _kernels as K
    inst = Instrument()
    cases = [('bench frame', bench_frame())]
    cases += [(f'{n} x {a} um', size_frame(a, n)) for a, n in FRAME_SIZES]
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    for name, p in cases:
        m = LorenzMie(coordinates=LorenzMie.meshgrid((1024, 1280)),
                      particle=spheres(p), instrument=inst)
        for _ in range(3):
            m.hologram(device=True)
        ts = []
        for _ in range(max(repeat, 1)):
            torch.cuda.synchronize()
            e0.record()
            m.hologram(device=True)
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        nmax = K.wiscombe_yang(p[:, 3], p[:, 4], p[:, 5], inst.n_m,
                               inst.wavelength)
        print(f'{name:14s} sum_nmax {int(nmax.sum()):5d} '
              f'{float(np.median(ts)):8.3f} ms')


if __name__ == '__main__':
    # python -m pylorenzmie_b200.workloads estimate_frame [--device-search]
    #     [--optimize]
    # python -m pylorenzmie_b200.workloads frame [--fp64]
    # python -m pylorenzmie_b200.workloads frame_sizes [--repeat N]
    # runs one workload through the public API, e.g. under a profiler
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument('workload', choices=['estimate_frame', 'frame',
                                         'frame_sizes'])
    ap.add_argument('--device-search', action='store_true')
    ap.add_argument('--repeat', type=int, default=2)
    ap.add_argument('--optimize', action='store_true')
    ap.add_argument('--fp64', action='store_true')
    a = ap.parse_args()
    if a.workload == 'frame':
        _run_frame(a.repeat, a.fp64)
    elif a.workload == 'frame_sizes':
        _run_frame_sizes(a.repeat)
    else:
        _run_estimate_frame(a.device_search, a.repeat, a.optimize)
