'''Multi-rank partitioning of fits and frames (pylorenzmie_b200.distributed)
on CPU: world_size-2 gloo process groups with stand-in per-rank work, so the
sharding, gathering and reassembly logic runs without a GPU.'''
import os
import socket

import numpy as np
import pandas as pd
import pytest

from pylorenzmie_b200 import distributed as D


def test_shard_features_balance_and_cover():
    rng = np.random.default_rng(1)
    costs = rng.integers(2500, 90000, 257) * rng.integers(17, 80, 257)
    for world in (1, 2, 3, 8):
        shares = D.shard_features(costs, world)
        assert len(shares) == world
        allidx = np.concatenate(shares)
        assert sorted(allidx) == list(range(257))
        loads = np.array([costs[s].sum() for s in shares])
        # LPT: within the largest single item of the mean
        assert loads.max() - loads.min() <= costs.max()
        assert all(np.all(np.diff(s) > 0) for s in shares)
    assert [len(s) for s in D.shard_features([5., 1.], 4)] == [1, 1, 0, 0]
    with pytest.raises(ValueError):
        D.shard_features([1.], 0)


def test_row_bands():
    assert D.row_bands(1024, 1) == [(0, 1024)]
    b = D.row_bands(1024, 3)
    assert b[0][0] == 0 and b[-1][1] == 1024
    assert all(b[i][1] == b[i + 1][0] for i in range(2))
    assert max(y - x for x, y in b) - min(y - x for x, y in b) <= 1
    b = D.row_bands(2, 4)
    assert sum(y - x for x, y in b) == 2 and b[0][0] == 0 and b[-1][1] == 2
    assert all(b[i][1] == b[i + 1][0] for i in range(3))


def test_feature_costs_scale_with_pixels_and_orders():
    starts = np.array([[0, 0, 100, 0.75, 1.42, 0], [0, 0, 100, 3.0, 1.7, 0]])
    c = D.feature_costs([1000, 1000], starts, 1.34, 0.447)
    assert c[1] > 2 * c[0]
    c2 = D.feature_costs([2000, 1000], starts, 1.34, 0.447)
    assert c2[0] == 2 * c[0]


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _stand_in_fit(seen):
    def fit(holos, particles, starts):
        seen.extend(int(h.data[0, 0]) for h in holos)
        return pd.DataFrame({'x_p': starts[:, 0] + 0.5, 'a_p': starts[:, 3],
                             'npix': [h.data.size for h in holos],
                             'success': True})
    return fit


def _worker(rank, world, port, queue):
    import torch.distributed as dist
    from pylorenzmie_b200 import Hologram, LorenzMie, Optimizer
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    from datetime import timedelta
    dist.init_process_group('gloo', rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    try:
        rng = np.random.default_rng(0)   # same inputs on every rank
        sides = rng.integers(20, 120, 23)
        holos = []
        for i, s in enumerate(sides):
            d = np.zeros((s, s))
            d[0, 0] = i                  # tags the feature
            holos.append(Hologram(d))
        starts = np.zeros((23, 6))
        starts[:, 0] = np.arange(23)
        starts[:, 2] = 150.
        starts[:, 3] = rng.uniform(0.5, 3.0, 23)
        starts[:, 4] = 1.45
        opt = Optimizer(model=LorenzMie(coordinates=np.zeros((2, 1))))
        seen = []
        df = D.optimize_batch_distributed(opt, holos, starts=starts,
                                          fit=_stand_in_fit(seen))
        frame = D.hologram_distributed(
            None, (37, 11),
            render=lambda m, rows: np.repeat(
                np.arange(rows[0], rows[1], dtype=float)[:, None], 11, 1))
        queue.put((rank, seen, df.to_dict('list'), frame.tolist()))
    finally:
        dist.destroy_process_group()


def test_two_rank_fit_and_frame_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context('spawn')
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, queue))
             for r in range(2)]
    for p in procs:
        p.start()
    out = [queue.get(timeout=180) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    seen0, seen1 = out[0][1], out[1][1]
    assert set(seen0).isdisjoint(seen1)
    assert sorted(seen0 + seen1) == list(range(23))
    assert seen0 and seen1
    for _, _, df, frame in out:          # every rank: the full result
        np.testing.assert_array_equal(df['x_p'], np.arange(23) + 0.5)
        assert len(df['npix']) == 23
        f = np.array(frame)
        np.testing.assert_array_equal(f[:, 0], np.arange(37))
        assert f.shape == (37, 11)
