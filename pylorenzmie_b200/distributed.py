'''Multi-GPU fitting and rendering: one process per GPU, no data-path
collective.

Features are independent Levenberg-Marquardt problems and a frame's pixels
are independent given the particle list, so the work partitions without any
exchange: every rank holds the same inputs, takes its own share, computes it
on its GPU, and the results (about 16 numbers per feature, or one band of
rows per rank) are gathered at the end -- the only communication, over the
process group's backend (NCCL on GPUs, gloo for host-only runs).  The
reference has no multi-GPU path; its batch loop is Frame.optimize
(analysis/Frame.py:163-174), one feature after another.

    import torch.distributed as dist
    dist.init_process_group('nccl')          # one process per GPU
    df = optimize_batch_distributed(optimizer, holograms, starts=starts)
    # every rank gets the full DataFrame, rows in input order
'''
import numpy as np
import pandas as pd

from .theory import _kernels as K


def feature_costs(npix, starts, n_m, wavelength):
    '''Work estimate of each feature: pixels x partial-wave orders at its
    start point (the evaluation kernel's cost is proportional to both).'''
    starts = np.asarray(starts, dtype=float).reshape(-1, 6)
    nmax = K.wiscombe_yang(starts[:, 3], starts[:, 4], starts[:, 5], n_m,
                           wavelength)
    return np.asarray(npix, dtype=float) * (nmax + 1.)


def shard_features(costs, world_size):
    '''Partition feature indices over ranks by estimated cost: longest
    processing time first (each feature, most expensive first, goes to the
    least-loaded rank).  Deterministic; returns a sorted index array per
    rank (some may be empty).'''
    if world_size < 1:
        raise ValueError('world_size must be at least 1')
    costs = np.asarray(costs, dtype=float)
    order = np.argsort(-costs, kind='stable')
    load = np.zeros(world_size)
    owner = np.empty(costs.size, dtype=np.int64)
    for i in order:
        r = int(np.argmin(load))  # lowest rank on ties
        owner[i] = r
        load[r] += costs[i]
    return [np.flatnonzero(owner == r) for r in range(world_size)]


def row_bands(ny, world_size):
    '''Contiguous row ranges [(start, stop)] of a frame, one per rank.'''
    if world_size < 1:
        raise ValueError('world_size must be at least 1')
    edges = np.linspace(0, ny, world_size + 1).round().astype(int)
    return [(int(a), int(b)) for a, b in zip(edges[:-1], edges[1:])]


def _group_info(group):
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return 0, 1
    return dist.get_rank(group), dist.get_world_size(group)


def _all_gather(obj, group, world):
    import torch.distributed as dist
    if world == 1:
        return [obj]
    out = [None] * world
    dist.all_gather_object(out, obj, group=group)
    return out


def optimize_batch_distributed(optimizer, holograms, particles=None,
                               starts=None, group=None, fit=None, **kwargs):
    '''Optimizer.optimize_batch over every rank of ``group`` (default: the
    world), each fitting its cost-balanced share of the features on its own
    GPU.  Every rank passes the same holograms and starts and receives the
    full result DataFrame in input order.  ``fit(holograms, particles,
    starts)`` replaces the per-rank fit (default: the optimizer's own
    optimize_batch with ``kwargs``).'''
    rank, world = _group_info(group)
    n = len(holograms)
    if fit is None:
        def fit(h, p, s):
            return optimizer.optimize_batch(h, particles=p, starts=s,
                                            **kwargs)
    if n == 0:  # the same on every rank: no collective
        return fit([], None, np.zeros((0, 6)))
    if starts is None:
        if particles is None:
            raise ValueError('give particles or starts')
        starts = np.array([[*(np.asarray(p.r_p, float) + np.asarray(
            getattr(p, 'r_0', (0., 0., 0.)), float)), p.a_p, p.n_p,
            getattr(p, 'k_p', 0.)] for p in particles], dtype=float)
    starts = np.asarray(starts, dtype=float).reshape(-1, 6)
    if starts.shape[0] != n:
        raise ValueError('one start per hologram')
    inst = optimizer.model.instrument
    npix = [np.asarray(optimizer._pixels(h)[0]).size for h in holograms]
    shares = shard_features(feature_costs(npix, starts, inst.n_m,
                                          inst.wavelength), world)
    mine = shares[rank]
    sub_particles = None if particles is None else [particles[i] for i in mine]
    if len(mine):
        part = fit([holograms[i] for i in mine], sub_particles, starts[mine])
    else:
        part = None
    gathered = _all_gather((mine, part), group, world)
    frames, index = [], []
    for idx, df in gathered:
        if df is not None and len(idx):
            frames.append(df.reset_index(drop=True))
            index.append(np.asarray(idx))
    out = pd.concat(frames, ignore_index=True)
    order = np.argsort(np.concatenate(index), kind='stable')
    return out.iloc[order].reset_index(drop=True)


def hologram_distributed(model, shape, group=None, render=None):
    '''The model's hologram of a full ny x nx frame (pixel grid at the
    origin), each rank rendering one band of rows on its GPU; every rank
    receives the whole (ny, nx) float64 frame.  ``render(model, rows)``
    replaces the per-rank band renderer (default: the model's own
    hologram() on the band's coordinates).'''
    from .lib import meshgrid
    rank, world = _group_info(group)
    ny, nx = shape
    a, b = row_bands(ny, world)[rank]
    if render is None:
        def render(m, rows):
            r0, r1 = rows
            if r1 <= r0:
                return np.zeros((0, nx))
            m.coordinates = meshgrid((r1 - r0, nx), corner=(0, r0))
            return np.asarray(m.hologram()).reshape(r1 - r0, nx)
    band = render(model, (a, b))
    bands = _all_gather(((a, b), np.asarray(band)), group, world)
    frame = np.empty((ny, nx))
    for (r0, r1), img in bands:
        frame[r0:r1] = img
    return frame


__all__ = ['feature_costs', 'shard_features', 'row_bands',
           'optimize_batch_distributed', 'hologram_distributed']
