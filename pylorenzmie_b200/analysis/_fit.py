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
        offs = self.features['data_offset']

        def work(lo, hi):
            for i in range(lo, hi):
                src = self._sources[i]
                n = src.size
                np.copyto(out[offs[i]:offs[i] + n], src.reshape(-1),
                          casting='unsafe')
        nf = len(self._sources)
        pool = _pool()
        if pool is None or self.total < (1 << 20) or nf < 4:
            work(0, nf)
            return out
        nthreads = pool._max_workers
        step = (nf + nthreads - 1) // nthreads
        futs = [pool.submit(work, lo, min(lo + step, nf))
                for lo in range(0, nf, step)]
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


def _pool():
    '''Thread pool for packing (numpy releases the GIL while copying).'''
    global _POOL
    if _POOL is None:
        import os
        from concurrent.futures import ThreadPoolExecutor
        n = min(16, os.cpu_count() or 1)
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


def upload(packed, starts, device=None):
    '''Device copies of a packed batch: (features, data, coords, params).
    The crops are converted to float32 directly into the pinned staging
    buffer and everything crosses to the device in one copy.'''
    dev = get_device(device)
    starts = np.ascontiguousarray(starts, dtype=np.float64).reshape(-1, 6)
    pieces = [packed.features.view(np.uint8), None, starts]
    if packed.coords is not None:
        pieces.append(packed.coords)
    nbytes = [packed.features.nbytes, packed.total * 4, starts.nbytes]
    if packed.coords is not None:
        nbytes.append(packed.coords.nbytes)
    sizes = [(n + 255) // 256 * 256 for n in nbytes]
    total = sum(sizes)
    stage = _staging.take(total)
    host = stage.numpy()
    offs = np.concatenate([[0], np.cumsum(sizes)[:-1]])
    for k, a in enumerate(pieces):
        if a is None:
            packed.write_data(host[offs[k]:offs[k] + nbytes[k]].view(np.float32))
        else:
            host[offs[k]:offs[k] + nbytes[k]] = a.view(np.uint8).reshape(-1)
    dbuf = torch.empty(max(total, 1), dtype=torch.uint8, device=dev)
    dbuf[:total].copy_(stage[:total], non_blocking=True)
    dtypes = [torch.uint8, torch.float32, torch.float64, torch.float32]
    out = [dbuf[offs[k]:offs[k] + nbytes[k]].view(dtypes[k])
           for k in range(len(pieces))]
    # the staging buffer is reused by the next call: wait for this copy
    torch.cuda.current_stream(dev).synchronize()
    d_coords = out[3] if packed.coords is not None else None
    return out[0], out[1], d_coords, out[2]


def fit_device(d_feat, d_data, d_coords, d_params, nfeatures, total_pixels,
               instrument, variables, settings=None, nmax_cap=None,
               starts_host=None, stats=False, tile_config=0, layers=None):
    '''Run lmb_fit_batch on device-resident inputs.  d_params is updated in
    place with the fitted values; returns (results tensor (B*80 uint8),
    FitStats or None).'''
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
    if layers is None:
        _native.check(lib.lmb_fit_batch(
            ptr(d_feat), nfeatures, total_pixels, ptr(d_data), ptr(d_coords),
            ptr(d_params), n_m, lam, float(instrument.magnification),
            float(instrument.noise), nmax_cap, st, ptr(d_res), ptr(ws),
            nbytes, fs, stream_handle(dev)), 'lmb_fit_batch')
        return d_res, fs
    L, frac, idx = layers
    d_frac = torch.from_numpy(np.ascontiguousarray(frac, dtype=np.float64)
                              ).to(dev)
    ind = np.zeros((nfeatures, L - 1, 2))
    ind[..., 0] = np.real(idx)
    ind[..., 1] = np.imag(idx)
    d_ind = torch.from_numpy(ind).to(dev)
    _native.check(lib.lmb_fit_batch_layered(
        ptr(d_feat), nfeatures, total_pixels, ptr(d_data), ptr(d_coords),
        ptr(d_params), L, ptr(d_frac), ptr(d_ind), n_m, lam,
        float(instrument.magnification), float(instrument.noise), nmax_cap,
        st, ptr(d_res), ptr(ws), nbytes, fs, stream_handle(dev)),
        'lmb_fit_batch_layered')
    return d_res, fs


def fit_packed(packed, starts, instrument, variables, settings=None,
               device=None, nmax_cap=None, stats=False, layers=None,
               autotune=False):
    '''Fit every packed feature; returns (params (B, 6), results record
    array with dparams, redchi, cost, status, success, nfev, njev) and,
    when stats, the FitStats of the call.'''
    starts = np.ascontiguousarray(starts, dtype=np.float64).reshape(-1, 6)
    B = starts.shape[0]
    if B == 0:
        res = np.zeros(0, dtype=_native.RESULT_DTYPE)
        return (starts.copy(), res, None) if stats else (starts.copy(), res)
    d_feat, d_data, d_coords, d_params = upload(packed, starts, device)
    if nmax_cap is None:
        nmax_cap = fit_capacity(starts, float(instrument.n_m),
                                float(instrument.wavelength), layers)
    tile_config = 0
    if autotune:
        from .. import autotune as _tuner
        tile_config = _tuner.tune(packed, starts, instrument, variables,
                                  nmax_cap, layers, d_data.device)
    d_res, fs = fit_device(d_feat, d_data, d_coords, d_params, B,
                           packed.total, instrument, variables, settings,
                           nmax_cap, starts, stats, tile_config=tile_config,
                           layers=layers)
    params = d_params.view(torch.float64).reshape(B, 6).cpu().numpy()
    res = d_res[:B * _native.RESULT_DTYPE.itemsize].cpu().numpy().view(
        _native.RESULT_DTYPE).copy()
    return (params, res, fs) if stats else (params, res)
