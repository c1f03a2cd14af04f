'''Host side of the batched device fit (``lmb_fit_batch``).

Packs crops of normalized holograms into one float32 buffer, copies it to
the device through pinned memory, runs every feature's Levenberg-Marquardt
fit in the CUDA library, and returns fitted parameters and statistics.
'''
import numpy as np
import torch

from .. import _native
from .._device import get_device, stream_handle, ptr
from ..theory import _kernels as K

PARAM_KEYS = ('x_p', 'y_p', 'z_p', 'a_p', 'n_p', 'k_p')
DEFAULT_SETTINGS = {'method': 'lm', 'ftol': 1e-4, 'xtol': 1e-6,
                    'gtol': 1e-6, 'loss': 'linear', 'max_nfev': 2000,
                    'diff_step': 1e-5, 'x_scale': 'jac'}


def variable_mask(variables):
    mask = 0
    for v in variables:
        mask |= 1 << PARAM_KEYS.index(v)
    return mask


def fit_capacity(starts, n_m, wavelength, layers=None):
    '''Partial-wave capacity for fits that start at ``starts`` (B, 6): room
    for a_p to grow 25 % and n_p by 0.25 during the fit.'''
    a = starts[:, 3] * 1.25
    n = starts[:, 4] + 0.25
    k = starts[:, 5]
    if layers is None:
        return K.nmax_cap_for(a, n, k, n_m, wavelength, margin=4)
    _, frac, idx = layers
    best = 0
    for i in range(starts.shape[0]):
        radii = np.append(frac[i] * a[i], a[i])
        ind = np.append(idx[i], n[i] + 1j * k[i])
        best = max(best, K.wiscombe_yang_layers(radii, ind, n_m, wavelength))
    cap = best + 4
    if cap > _native.LMB_NMAX_LIMIT:
        raise ValueError(f'a sphere needs {best} partial-wave orders; the '
                         f'limit is {_native.LMB_NMAX_LIMIT}')
    return cap


def layers_of(particles):
    '''(nlayers, fractions (B, L-1), inner indices (B, L-1) complex) of a
    list of LayeredSphere particles with one layer count, or None.'''
    if not particles or not K.is_layered(particles[0]):
        return None
    L = particles[0].nlayers
    if any(not K.is_layered(p) or p.nlayers != L for p in particles):
        raise ValueError('a batch fits spheres with one layer count')
    frac = np.array([p.fractions for p in particles], dtype=float)
    idx = np.array([p.core_indices for p in particles], dtype=complex)
    return L, frac.reshape(len(particles), L - 1), \
        idx.reshape(len(particles), L - 1)


class PackedFeatures:
    '''Crops packed for the device: float32 data, lmb_feature records and
    optional float32 (x, y) coordinates for non-grid pixel sets.

    The crops are not copied here: ``write_data`` converts them straight
    into a destination buffer (the pinned staging buffer of ``upload``),
    in parallel over features; ``data`` builds a host copy on demand.
    '''

    def __init__(self, items):
        '''items: list of (data, grid, coords): data (npix,) or (ny, nx);
        grid (x0, y0, ny, nx), or None with explicit coords (2, npix).'''
        feats = np.zeros(len(items), dtype=_native.FEATURE_DTYPE)
        self._sources = []
        cchunks = []
        off = 0
        explicit = any(it[1] is None for it in items)
        for i, (data, grid, coords) in enumerate(items):
            d = np.asarray(data)
            n = d.size
            if grid is not None:
                x0, y0, ny, nx = grid
                if ny * nx != n:
                    raise ValueError('data size does not match its grid')
                feats[i] = (x0, y0, nx, ny, n, off)
            else:
                feats[i] = (0., 0., 0, 0, n, off)
            self._sources.append(d)
            if explicit:
                if grid is None:
                    c = np.asarray(coords, dtype=np.float32)[:2].T
                else:
                    x0, y0, ny, nx = grid
                    yy, xx = np.mgrid[0:ny, 0:nx]
                    c = np.stack([x0 + xx.ravel(), y0 + yy.ravel()], axis=1
                                 ).astype(np.float32)
                cchunks.append(np.ascontiguousarray(c))
            off += n
        self.features = feats
        self.coords = (np.concatenate(cchunks).reshape(-1)
                       if explicit and cchunks else None)
        self.total = off
        self._data = None

    def write_data(self, out):
        '''Convert every crop into the float32 array ``out`` (total,).'''
        return self.write_range(out, 0, len(self._sources))

    def write_range(self, out, lo, hi):
        '''Convert crops lo..hi-1 into their places in ``out`` (total,).
        The crops are contiguous in ``out``; the range is cut into equal
        runs of pixels, one per thread, whatever the crop sizes.  Float64
        or float32 crops are converted by the library's native threads
        (lmb_pack_crops), others by numpy.'''
        if hi <= lo:
            return out
        offs = self.features['data_offset']
        npix = self.features['npix']
        begin = int(offs[lo])
        end = int(offs[hi - 1] + npix[hi - 1])
        srcs = self._sources[lo:hi]
        kind = _pack_kind(srcs)
        if kind is not None and out.dtype == np.float32 and \
                out.flags.c_contiguous:
            ptrs = np.array([s.ctypes.data for s in srcs], dtype=np.uintp)
            counts = np.ascontiguousarray(npix[lo:hi], dtype=np.int64)
            _native.check(_native.load().lmb_pack_crops(
                ptrs.ctypes.data, counts.ctypes.data, hi - lo, kind,
                out[begin:].ctypes.data, _pack_threads()), 'lmb_pack_crops')
            return out

        def work(a, b):  # pixels [a, b) of the packed buffer
            i = int(np.searchsorted(offs, a, side='right')) - 1
            while a < b:
                n0 = int(offs[i])
                n = int(npix[i])
                s0, s1 = a - n0, min(b, n0 + n) - n0
                if s1 > s0:
                    np.copyto(out[n0 + s0:n0 + s1],
                              self._sources[i].reshape(-1)[s0:s1],
                              casting='unsafe')
                a = n0 + s1 if s1 > s0 else a
                i += 1
        pool = _pool()
        if pool is None or end - begin < (1 << 19):
            work(begin, end)
            return out
        nthreads = pool._max_workers
        cuts = np.linspace(begin, end, nthreads + 1).astype(np.int64)
        futs = [pool.submit(work, int(a), int(b))
                for a, b in zip(cuts[:-1], cuts[1:]) if b > a]
        for f in futs:
            f.result()
        return out

    @property
    def data(self):
        if self._data is None:
            self._data = self.write_data(np.empty(self.total, np.float32))
        return self._data

    @property
    def h2d_bytes(self):
        n = self.total * 4 + self.features.nbytes
        if self.coords is not None:
            n += self.coords.nbytes
        return n


_POOL = None


def _pack_kind(sources):
    '''LMB_PACK_F64/F32 if every source is a C-contiguous array of that
    type, else None.'''
    if not sources:
        return None
    dt = sources[0].dtype
    kinds = {np.dtype(np.float64): _native.LMB_PACK_F64,
             np.dtype(np.float32): _native.LMB_PACK_F32}
    if dt not in kinds:
        return None
    if any(s.dtype != dt or not s.flags.c_contiguous for s in sources):
        return None
    return kinds[dt]


def _pack_threads():
    import os
    # leave a core for the thread that drives a streamed fit (its waits on
    # the GPU spin)
    return max(1, min(32, (os.cpu_count() or 1) - 1))




def _pool():
    '''Thread pool for packing (numpy releases the GIL while copying).'''
    global _POOL
    if _POOL is None:
        import os
        from concurrent.futures import ThreadPoolExecutor
        # leave a core each for the caller and the thread that drives a
        # streamed fit (its waits on the GPU spin)
        n = min(16, (os.cpu_count() or 1) - 2)
        _POOL = ThreadPoolExecutor(max_workers=n) if n > 1 else False
    return _POOL or None


class _Staging:
    '''Reusable pinned host buffer for host-to-device copies (allocating
    pinned memory on every call would cost more than the copy).'''

    def __init__(self):
        self.buf = None

    def take(self, nbytes):
        if self.buf is None or self.buf.numel() < nbytes:
            self.buf = torch.empty(max(nbytes, 1 << 20), dtype=torch.uint8,
                                   pin_memory=True)
        return self.buf


_staging = _Staging()


def stage(packed, starts, staging=None):
    '''Write a packed batch into a pinned staging buffer: the crops as
    float32, the feature records, the starts and any explicit coordinates,
    each at a 256-byte aligned offset.  Returns (pinned uint8 tensor, offsets,
    sizes).'''
    starts = np.ascontiguousarray(starts, dtype=np.float64).reshape(-1, 6)
    pieces = [packed.features.view(np.uint8), None, starts]
    if packed.coords is not None:
        pieces.append(packed.coords)
    nbytes = [packed.features.nbytes, packed.total * 4, starts.nbytes]
    if packed.coords is not None:
        nbytes.append(packed.coords.nbytes)
    sizes = [(n + 255) // 256 * 256 for n in nbytes]
    total = sum(sizes)
    buf = (staging or _staging).take(total)
    host = buf.numpy()
    offs = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(int)
    for k, a in enumerate(pieces):
        if a is None:
            packed.write_data(host[offs[k]:offs[k] + nbytes[k]].view(np.float32))
        else:
            host[offs[k]:offs[k] + nbytes[k]] = a.view(np.uint8).reshape(-1)
    return buf, offs, nbytes


def to_device(buf, offs, nbytes, dev):
    '''One asynchronous copy of a staged batch on the current stream;
    device views (features, data, coords or None, params).  The pinned
    buffer must not be rewritten before the copy has completed.'''
    total = int(offs[-1] + (nbytes[-1] + 255) // 256 * 256)
    dbuf = torch.empty(max(total, 1), dtype=torch.uint8, device=dev)
    dbuf[:total].copy_(buf[:total], non_blocking=True)
    dtypes = [torch.uint8, torch.float32, torch.float64, torch.float32]
    out = [dbuf[offs[k]:offs[k] + nbytes[k]].view(dtypes[k])
           for k in range(len(nbytes))]
    d_coords = out[3] if len(nbytes) > 3 else None
    return out[0], out[1], d_coords, out[2]


def upload(packed, starts, device=None):
    '''Device copies of a packed batch: (features, data, coords, params).
    The crops are converted to float32 directly into the pinned staging
    buffer and everything crosses to the device in one copy.'''
    dev = get_device(device)
    buf, offs, nbytes = stage(packed, starts)
    out = to_device(buf, offs, nbytes, dev)
    # the staging buffer is reused by the next call: wait for this copy
    torch.cuda.current_stream(dev).synchronize()
    return out


def fit_device(d_feat, d_data, d_coords, d_params, nfeatures, total_pixels,
               instrument, variables, settings=None, nmax_cap=None,
               starts_host=None, stats=False, tile_config=0, layers=None,
               ready=None, wait_seconds=60., aberration=0.):
    '''Run lmb_fit_batch on device-resident inputs.  d_params is updated in
    place with the fitted values; returns (results tensor (B*80 uint8),
    FitStats or None).  With ``ready`` (a device int32 tensor) the fit is
    streamed (lmb_fit_batch_streamed): features are admitted as the caller
    advances it.  A nonzero ``aberration`` (the coefficient c of the
    spherical-aberration phase, AberratedLorenzMie._aberration) fits the
    aberrated model (lmb_fit_batch_aberrated, or lmb_fit_batch_streamed
    with the coefficient).'''
    dev = d_data.device
    lib = _native.load()
    settings = dict(DEFAULT_SETTINGS if settings is None else settings)
    n_m = float(instrument.n_m)
    lam = float(instrument.wavelength)
    if nmax_cap is None:
        sh = (starts_host if starts_host is not None
              else d_params.view(torch.float64).reshape(-1, 6).cpu().numpy())
        nmax_cap = fit_capacity(sh, n_m, lam)
    d_res = torch.empty(max(nfeatures, 1) * _native.RESULT_DTYPE.itemsize,
                        dtype=torch.uint8, device=dev)
    nbytes = lib.lmb_fit_workspace_bytes(nfeatures, total_pixels, nmax_cap)
    ws = torch.empty(max(nbytes, 1), dtype=torch.uint8, device=dev)
    st = _native.FitSettings()
    st.ftol = float(settings.get('ftol', 1e-4) or 0.)
    st.xtol = float(settings.get('xtol', 1e-6) or 0.)
    st.gtol = float(settings.get('gtol', 1e-6) or 0.)
    st.factor = 100.
    st.max_nfev = int(settings.get('max_nfev', 2000) or 2000)
    st.variables = variable_mask(variables)
    st.flags = _native.LMB_BOHREN
    st.max_iterations = st.max_nfev
    st.tile_config = int(tile_config)
    fs = _native.FitStats() if stats else None
    if aberration and ready is None:
        if layers is None:
            L, d_frac, d_ind = 1, None, None
        else:
            L, d_frac, d_ind = _layer_arrays(layers, nfeatures, dev)
        _native.check(lib.lmb_fit_batch_aberrated(
            ptr(d_feat), nfeatures, total_pixels, ptr(d_data), ptr(d_coords),
            ptr(d_params), L, ptr(d_frac), ptr(d_ind), n_m, lam,
            float(instrument.magnification), float(instrument.noise),
            nmax_cap, float(aberration), st, ptr(d_res), ptr(ws), nbytes, fs,
            stream_handle(dev)), 'lmb_fit_batch_aberrated')
        return d_res, fs
    if ready is not None:
        if layers is None:
            L, d_frac, d_ind = 1, None, None
        else:
            L, d_frac, d_ind = _layer_arrays(layers, nfeatures, dev)
        _native.check(lib.lmb_fit_batch_streamed(
            ptr(d_feat), nfeatures, total_pixels, ptr(d_data), ptr(d_coords),
            ptr(d_params), L, ptr(d_frac), ptr(d_ind), n_m, lam,
            float(instrument.magnification), float(instrument.noise),
            nmax_cap, st, ptr(ready), float(wait_seconds), ptr(d_res),
            ptr(ws), nbytes, fs, stream_handle(dev), float(aberration)),
            'lmb_fit_batch_streamed')
        return d_res, fs
    if layers is None:
        _native.check(lib.lmb_fit_batch(
            ptr(d_feat), nfeatures, total_pixels, ptr(d_data), ptr(d_coords),
            ptr(d_params), n_m, lam, float(instrument.magnification),
            float(instrument.noise), nmax_cap, st, ptr(d_res), ptr(ws),
            nbytes, fs, stream_handle(dev)), 'lmb_fit_batch')
        return d_res, fs
    L, d_frac, d_ind = _layer_arrays(layers, nfeatures, dev)
    _native.check(lib.lmb_fit_batch_layered(
        ptr(d_feat), nfeatures, total_pixels, ptr(d_data), ptr(d_coords),
        ptr(d_params), L, ptr(d_frac), ptr(d_ind), n_m, lam,
        float(instrument.magnification), float(instrument.noise), nmax_cap,
        st, ptr(d_res), ptr(ws), nbytes, fs, stream_handle(dev)),
        'lmb_fit_batch_layered')
    return d_res, fs


def _layer_arrays(layers, nfeatures, dev):
    '''(nlayers, device fractions, device inner indices (re, im)).'''
    L, frac, idx = layers
    d_frac = torch.from_numpy(np.ascontiguousarray(frac, dtype=np.float64)
                              ).to(dev)
    ind = np.zeros((nfeatures, L - 1, 2))
    ind[..., 0] = np.real(idx)
    ind[..., 1] = np.imag(idx)
    d_ind = torch.from_numpy(ind).to(dev)
    return L, d_frac, d_ind


# Launch shape of the evaluation kernel (lmb_fit_tile_config index) for
# batches that are not autotuned.  A batch of fewer than SMALL_BATCH
# features has few 512-pixel tiles per round, and the round is latency-
# bound: SMALL_SHAPE (256 threads x one pixel pair) keeps each thread's
# chain of pixels short.  Measured on a B200 against the default shape 0
# (64 threads x 8 pixels): Frame.optimize of 32 features of 121x121 px
# 6.56 -> 6.21 ms, one 201x201 fit 1.40 -> 1.22 ms, 32 three-layer features
# 9.5 -> 8.3 ms.  Larger batches keep shape 0 or the autotuner's choice.
# The shape fixes the order of each tile's sums, so fits of the same
# features in batches of either kind differ in the last bits.
SMALL_BATCH = 64
SMALL_SHAPE = 7


def default_shape(nfeatures):
    '''Evaluation shape of a batch of nfeatures that is not autotuned.'''
    return SMALL_SHAPE if nfeatures < SMALL_BATCH else 0


def fit_packed(packed, starts, instrument, variables, settings=None,
               device=None, nmax_cap=None, stats=False, layers=None,
               autotune=False, aberration=0.):
    '''Fit every packed feature; returns (params (B, 6), results record
    array with dparams, redchi, cost, status, success, nfev, njev) and,
    when stats, the FitStats of the call.  ``aberration``: see fit_device.'''
    starts = np.ascontiguousarray(starts, dtype=np.float64).reshape(-1, 6)
    B = starts.shape[0]
    if B == 0:
        res = np.zeros(0, dtype=_native.RESULT_DTYPE)
        return (starts.copy(), res, None) if stats else (starts.copy(), res)
    d_feat, d_data, d_coords, d_params = upload(packed, starts, device)
    if nmax_cap is None:
        nmax_cap = fit_capacity(starts, float(instrument.n_m),
                                float(instrument.wavelength), layers)
    tile_config = default_shape(B)
    if autotune and not aberration:   # the aberrated fit has one shape
        from .. import autotune as _tuner
        tile_config = _tuner.tune(packed, starts, instrument, variables,
                                  nmax_cap, layers, d_data.device)
    d_res, fs = fit_device(d_feat, d_data, d_coords, d_params, B,
                           packed.total, instrument, variables, settings,
                           nmax_cap, starts, stats, tile_config=tile_config,
                           layers=layers, aberration=aberration)
    params = d_params.view(torch.float64).reshape(B, 6).cpu().numpy()
    res = d_res[:B * _native.RESULT_DTYPE.itemsize].cpu().numpy().view(
        _native.RESULT_DTYPE).copy()
    return (params, res, fs) if stats else (params, res)


_streams = {}


def _fit_streams(dev):
    '''(fit stream, copy stream) of a device, created once.'''
    if dev not in _streams:
        _streams[dev] = (torch.cuda.Stream(dev), torch.cuda.Stream(dev))
    return _streams[dev]


_flags = None
_WORKER = None


def _worker():
    global _WORKER
    if _WORKER is None:
        from concurrent.futures import ThreadPoolExecutor
        _WORKER = ThreadPoolExecutor(max_workers=1)
    return _WORKER


def default_chunks(npix):
    '''Portions in which a batch's pixel data is streamed to the device:
    one below ~2 Mpx (the host work is short), else up to 8 of at least
    ~1 Mpx each.'''
    total = int(np.sum(npix))
    if len(npix) < 8 or total < (2 << 20):
        return 1
    return int(min(8, len(npix) // 4, total // (1 << 20)))


def split_by_pixels(npix, chunks):
    '''Contiguous index ranges with about equal pixel totals.'''
    cum = np.cumsum(npix)
    edges = [0]
    for c in range(1, chunks):
        edges.append(int(np.searchsorted(cum, cum[-1] * c / chunks)) + 1)
    edges.append(len(npix))
    edges = sorted(set(min(max(e, 0), len(npix)) for e in edges))
    return [(a, b) for a, b in zip(edges[:-1], edges[1:]) if b > a]


def fit_items(items, starts, instrument, variables, settings=None,
              device=None, layers=None, autotune=False, chunks=None,
              wait_seconds=60., aberration=0.):
    '''Fit crops given as (data, grid, coords) items.  Large batches are
    streamed: the feature records and starts go to the device first and the
    fit starts (lmb_fit_batch_streamed, driven by a worker thread); the host
    then converts the pixel data portion by portion into pinned memory and
    copies each on a second stream, advancing the device's admission count
    after each copy, so that conversion and transfer overlap the fitting of
    the features already admitted.  ``aberration``: see fit_device.
    Returns (params (B, 6), results record array, npix (B,)).'''
    global _flags
    starts = np.ascontiguousarray(starts, dtype=np.float64).reshape(-1, 6)
    B = starts.shape[0]
    if len(items) != B:
        raise ValueError('one start per feature')
    packed = PackedFeatures(items)
    npix = packed.features['npix'].astype(np.int64)
    if chunks is None:
        chunks = default_chunks(npix)
    if B == 0 or chunks <= 1:
        params, res = fit_packed(packed, starts, instrument, variables,
                                 settings, device, layers=layers,
                                 autotune=autotune, aberration=aberration)
        return params, res, npix
    dev = get_device(device)
    nmax_cap = fit_capacity(starts, float(instrument.n_m),
                            float(instrument.wavelength), layers)
    tile_config = default_shape(B)
    if autotune and not aberration:   # the aberrated fit has one shape
        from .. import autotune as _tuner
        tile_config = _tuner.tune(packed, starts, instrument, variables,
                                  nmax_cap, layers, dev)
    ranges = split_by_pixels(npix, chunks)
    # pinned layout: [features | starts | coords | data], 256-byte aligned
    pieces = [packed.features.view(np.uint8), starts.view(np.uint8)]
    if packed.coords is not None:
        pieces.append(packed.coords.view(np.uint8))
    sizes = [(p.nbytes + 255) // 256 * 256 for p in pieces]
    head = sum(sizes)
    total = head + packed.total * 4
    buf = _staging.take(total)
    host = buf.numpy()
    off = 0
    for p, sz in zip(pieces, sizes):
        host[off:off + p.nbytes] = p.reshape(-1)
        off += sz
    hdata = host[head:head + packed.total * 4].view(np.float32)
    if _flags is None or _flags.numel() < len(ranges) + 1:
        _flags = torch.zeros(max(len(ranges) + 1, 64), dtype=torch.int32,
                             pin_memory=True)
    s_fit, s_copy = _fit_streams(dev)
    s_fit.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(s_fit):
        dbuf = torch.empty(total, dtype=torch.uint8, device=dev)
        dbuf[:head].copy_(buf[:head], non_blocking=True)
        d_ready = torch.zeros(1, dtype=torch.int32, device=dev)
    s_copy.wait_stream(s_fit)
    dbuf.record_stream(s_copy)
    d_ready.record_stream(s_copy)
    d_feat = dbuf[:pieces[0].nbytes]
    d_params = dbuf[sizes[0]:sizes[0] + pieces[1].nbytes].view(torch.float64)
    d_coords = None
    if packed.coords is not None:
        o = sizes[0] + sizes[1]
        d_coords = dbuf[o:o + pieces[2].nbytes].view(torch.float32)
    d_data = dbuf[head:total].view(torch.float32)
    future = _worker().submit(_fit_streamed, s_fit, d_feat, d_data, d_coords,
                              d_params, B, packed.total, instrument,
                              variables, settings, nmax_cap, starts,
                              tile_config, layers, d_ready, wait_seconds,
                              aberration)
    offs = packed.features['data_offset']
    try:
        for k, (a, b) in enumerate(ranges):
            packed.write_range(hdata, a, b)
            lo = int(offs[a]) * 4
            hi = int(offs[b - 1] + npix[b - 1]) * 4
            with torch.cuda.stream(s_copy):
                dbuf[head + lo:head + hi].copy_(buf[head + lo:head + hi],
                                                non_blocking=True)
                _flags[k] = b
                d_ready.copy_(_flags[k:k + 1], non_blocking=True)
    except BaseException:
        _flags[len(ranges)] = -1
        with torch.cuda.stream(s_copy):
            d_ready.copy_(_flags[len(ranges):len(ranges) + 1],
                          non_blocking=True)
        try:
            future.result()
        finally:
            s_copy.synchronize()
        raise
    try:
        params, res = future.result()
    finally:
        # the pinned buffers are reused by the next call
        s_copy.synchronize()
    torch.cuda.current_stream(dev).wait_stream(s_fit)
    return params, res, npix


def _fit_streamed(stream, d_feat, d_data, d_coords, d_params, n, total,
                  instrument, variables, settings, nmax_cap, starts,
                  tile_config, layers, d_ready, wait_seconds, aberration=0.):
    with torch.cuda.stream(stream):
        d_res, _ = fit_device(d_feat, d_data, d_coords, d_params, n, total,
                              instrument, variables, settings, nmax_cap,
                              starts, False, tile_config=tile_config,
                              layers=layers, ready=d_ready,
                              wait_seconds=wait_seconds, aberration=aberration)
        params = d_params.view(torch.float64).reshape(n, 6).cpu().numpy()
        res = d_res[:n * _native.RESULT_DTYPE.itemsize].cpu().numpy().view(
            _native.RESULT_DTYPE).copy()
    return params, res


_stream_staging = []
_STREAM_WORKER = None


_stream_fit_streams = {}


def _stream_worker(n):
    '''Threads that drive the fits of fit_stream, one per batch in flight:
    two consecutive fits run on different streams, so the kernels of one
    fill the GPU while the other waits on its host round trip.'''
    global _STREAM_WORKER
    if _STREAM_WORKER is None or _STREAM_WORKER._max_workers < n:
        from concurrent.futures import ThreadPoolExecutor
        old = _STREAM_WORKER
        _STREAM_WORKER = ThreadPoolExecutor(max_workers=n)
        if old is not None:
            # its threads end once the fits already given to them return
            old.shutdown(wait=False)
    return _STREAM_WORKER


def _stream_fit_stream(dev, slot):
    key = (dev, slot)
    if key not in _stream_fit_streams:
        _stream_fit_streams[key] = torch.cuda.Stream(dev)
    return _stream_fit_streams[key]


class _Slots:
    '''The scheduling of fit_stream: at most ``depth`` jobs run at once,
    each on a slot of its own (a stream); a slot frees when any job ends;
    results leave in submission order, with at most ``backlog`` finished
    ones held back.  ``wait_slot()`` blocks until a slot is free;
    ``submit(fn, extra, *args)`` takes it and calls fn(slot, *args) ->
    future; ``ready()`` yields the results whose turn has come (and the
    oldest ones past the backlog bound, waiting for them); ``drain()``
    yields the rest.  ``add_done(extra)`` queues a result that needs no job
    (an empty batch); it passes through as ``extra``.'''

    def __init__(self, depth, backlog=None):
        from collections import deque
        self.depth = depth
        self.backlog = 8 * depth if backlog is None else backlog
        self.pending = deque()      # (future or None, extra)
        self.running = {}           # future -> slot
        self.free = list(range(depth))

    def add_done(self, extra):
        self.pending.append((None, extra))

    def wait_slot(self):
        from concurrent.futures import wait, FIRST_COMPLETED
        while not self.free:
            finished, _ = wait(list(self.running),
                               return_when=FIRST_COMPLETED)
            for f in finished:
                self.free.append(self.running.pop(f))

    def ready(self):
        while self.pending and (self.pending[0][0] is None or
                                self.pending[0][0].done()):
            yield _collect(self.pending.popleft())
        while len(self.pending) >= self.backlog:
            yield _collect(self.pending.popleft())

    def submit(self, fn, extra, *args):
        slot = self.free.pop(0)
        fut = fn(slot, *args)
        self.running[fut] = slot
        self.pending.append((fut, extra))
        return slot

    def drain(self):
        while self.pending:
            yield _collect(self.pending.popleft())

    def wait_all(self):
        for fut, _ in self.pending:
            if fut is not None:
                fut.result()


def fit_stream(batches, instrument, variables, settings=None, device=None,
               autotune=False, depth=2, aberration=0.):
    '''Fit a sequence of batches, pipelined; yields, in order, (params
    (B, 6), results record array, npix (B,)) per batch.

    ``batches`` yields (items, starts, layers): items as for fit_items.
    Up to ``depth`` fits run at once, each driven by a worker thread on a
    stream of its own (consecutive fits overlap on the GPU).  The caller's
    thread converts the next batch into one of depth + 1 pinned buffers and
    copies it on the copy stream before it waits for a fit slot, so that
    batch's data is on the device when a slot frees; its fit waits for that
    copy on the device, not on the host.  A slot frees when any running fit
    ends, not only the oldest, so a batch whose slowest fit takes many
    rounds holds one slot while later batches pass through the others;
    finished batches wait, up to 8 x depth of them, to be yielded in order.
    A pinned buffer is rewritten only after its previous copy has
    completed.'''
    dev = get_device(device)
    _, s_copy = _fit_streams(dev)
    nstage = depth + 1
    while len(_stream_staging) < nstage:
        _stream_staging.append(_Staging())
    slots = _Slots(depth)
    done_events = [None] * nstage
    tile_config = None
    k = 0

    def launch(fit_slot, ev, views, B, total, nmax_cap, starts, layers):
        s_fit = _stream_fit_stream(dev, fit_slot)
        for v in views:
            if v is not None:
                v.record_stream(s_fit)
        return _stream_worker(depth).submit(
            _fit_after, s_fit, ev, views, B, total, instrument, variables,
            settings, nmax_cap, starts, tile_config, layers, aberration)

    try:
        for items, starts, layers in batches:
            starts = np.ascontiguousarray(starts, dtype=np.float64
                                          ).reshape(-1, 6)
            B = starts.shape[0]
            packed = PackedFeatures(items)
            npix = packed.features['npix'].astype(np.int64)
            if B == 0:
                slots.add_done((starts.copy(), np.zeros(
                    0, dtype=_native.RESULT_DTYPE), npix))
                k += 1
                continue
            nmax_cap = fit_capacity(starts, float(instrument.n_m),
                                    float(instrument.wavelength), layers)
            if tile_config is None:
                tile_config = default_shape(B)
                if autotune and not aberration:
                    from .. import autotune as _tuner
                    tile_config = _tuner.tune(packed, starts, instrument,
                                              variables, nmax_cap, layers,
                                              dev)
            slot = k % nstage
            if done_events[slot] is not None:
                done_events[slot].synchronize()  # its last copy has landed
            buf, offs, nbytes = stage(packed, starts, _stream_staging[slot])
            with torch.cuda.stream(s_copy):
                views = to_device(buf, offs, nbytes, dev)
                ev = torch.cuda.Event()
                ev.record(s_copy)
            done_events[slot] = ev
            # this batch's data is on its way: now wait for a fit slot
            slots.wait_slot()
            yield from slots.ready()
            slots.submit(launch, npix, ev, views, B, packed.total, nmax_cap,
                         starts, layers)
            k += 1
        yield from slots.drain()
    finally:
        slots.wait_all()
        s_copy.synchronize()


def _collect(entry):
    fut, extra = entry
    if fut is None:
        return extra
    params, res = fut.result()
    return params, res, extra


def _fit_after(stream, event, views, n, total, instrument, variables,
               settings, nmax_cap, starts, tile_config, layers, aberration=0.):
    d_feat, d_data, d_coords, d_params = views
    stream.wait_event(event)
    with torch.cuda.stream(stream):
        d_res, _ = fit_device(d_feat, d_data, d_coords, d_params, n, total,
                              instrument, variables, settings, nmax_cap,
                              starts, False, tile_config=tile_config,
                              layers=layers, aberration=aberration)
        params = d_params.view(torch.float64).reshape(n, 6).cpu().numpy()
        res = d_res[:n * _native.RESULT_DTYPE.itemsize].cpu().numpy().view(
            _native.RESULT_DTYPE).copy()
    return params, res
