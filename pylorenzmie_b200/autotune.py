'''Autotuner for the launch shape of the fit's evaluation kernel.

The evaluation kernel exists in several launch shapes (threads per CTA,
pixels per thread, register cap, CTA- or warp-granular tiles; see
``lmb_fit_tile_config``).  For a problem class -- partial-wave capacity
bucket and mean crop size bucket, on one GPU model -- the tuner times every
shape on a probe batch cut from the caller's own features (device time of
the evaluation launches, measured by the library with CUDA events) and
keeps the fastest.  Results are cached in memory and in a JSON file
(``$LMB200_AUTOTUNE_CACHE`` or ``~/.cache/pylorenzmie_b200/autotune.json``).
'''
import ctypes
import json
import os
import threading
from pathlib import Path

import numpy as np

from . import _native

_lock = threading.Lock()
_memory = {}
# the probe batch: up to PROBE_FEATURES of the caller's features (a shape
# that is fastest on a few features need not be on a full batch, whose
# tiles fill the GPU differently, so the batch size is part of the class)
PROBE_FEATURES = 256
NMAX_BUCKETS = (32, 64, 128, 256, 1024)
PIXEL_BUCKETS = (64 * 64, 128 * 128, 256 * 256, 512 * 512)
BATCH_BUCKETS = (64, 256)


def cache_path():
    env = os.environ.get('LMB200_AUTOTUNE_CACHE')
    if env:
        return Path(env)
    return Path.home() / '.cache' / 'pylorenzmie_b200' / 'autotune.json'


def shapes():
    '''List of (index, threads, pixels_per_thread, min_blocks).'''
    lib = _native.load()
    out = []
    i = 0
    while True:
        t, p, m = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        if lib.lmb_fit_tile_config(i, ctypes.byref(t), ctypes.byref(p),
                                   ctypes.byref(m)) != _native.LMB_OK:
            return out
        out.append((i, t.value, p.value, m.value))
        i += 1


def _bucket(value, edges):
    for e in edges:
        if value <= e:
            return e
    return edges[-1] * 2


def problem_key(gpu_name, nmax_cap, mean_pixels, layered=False,
                batch=PROBE_FEATURES):
    return (f'{gpu_name}|nmax<={_bucket(nmax_cap, NMAX_BUCKETS)}|'
            f'px<={_bucket(mean_pixels, PIXEL_BUCKETS)}|'
            f'b<={_bucket(batch, BATCH_BUCKETS)}|'
            f'{"layered" if layered else "sphere"}')


def _load_file():
    try:
        return json.loads(cache_path().read_text())
    except Exception:
        return {}


def _store(key, entry):
    path = cache_path()
    try:
        path.parent.mkdir(parents=True, exist_ok=True)
        data = _load_file()
        data[key] = entry
        # one temporary file per process: ranks on one host may store at once
        tmp = path.with_suffix(f'.{os.getpid()}.tmp')
        tmp.write_text(json.dumps(data, indent=1, sort_keys=True))
        tmp.replace(path)
    except OSError:
        pass  # a read-only home still tunes, per process


def lookup(key):
    with _lock:
        if key in _memory:
            return _memory[key]
        entry = _load_file().get(key)
        if entry is not None:
            _memory[key] = entry
        return entry


def tune(packed, starts, instrument, variables, nmax_cap, layers=None,
         device=None, repeats=2):
    '''Best shape index for this batch's problem class (timed if unknown).'''
    import torch
    from .analysis import _fit
    dev = device if device is not None else torch.device('cuda')
    name = torch.cuda.get_device_name(dev)
    B = packed.features.shape[0]
    mean_px = float(packed.features['npix'].mean()) if B else 0.
    key = problem_key(name, nmax_cap, mean_px, layers is not None, B)
    hit = lookup(key)
    if hit is not None:
        return int(hit['config'])
    n = min(B, PROBE_FEATURES)
    idx = np.arange(n)
    items = [(packed._sources[i],
              (packed.features['x0'][i], packed.features['y0'][i],
               packed.features['ny'][i], packed.features['nx'][i])
              if packed.features['nx'][i] > 0 else None,
              packed.coords.reshape(-1, 2)[
                  packed.features['data_offset'][i]:
                  packed.features['data_offset'][i] +
                  packed.features['npix'][i]].T
              if packed.features['nx'][i] == 0 else None) for i in idx]
    probe = _fit.PackedFeatures(items)
    sub_layers = None
    if layers is not None:
        sub_layers = (layers[0], layers[1][:n], layers[2][:n])
    d_feat, d_data, d_coords, d_params = _fit.upload(probe, starts[:n], dev)
    p0 = d_params.clone()
    timings = {}
    for (i, _, _, _) in shapes():
        best = None
        for _ in range(repeats):
            d_params.copy_(p0)
            _, fs = _fit.fit_device(d_feat, d_data, d_coords, d_params, n,
                                    probe.total, instrument, variables, None,
                                    nmax_cap, starts[:n], stats=True,
                                    tile_config=i, layers=sub_layers)
            per = fs.eval_ms / max(fs.eval_launches, 1)
            best = per if best is None else min(best, per)
        timings[i] = best
    choice = min(timings, key=timings.get)
    entry = {'config': int(choice),
             'eval_ms': {str(k): float(v) for k, v in timings.items()}}
    with _lock:
        _memory[key] = entry
    _store(key, entry)
    return int(choice)
