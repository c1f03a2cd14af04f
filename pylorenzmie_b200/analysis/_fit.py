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


def fit_capacity(starts, n_m, wavelength):
    '''Partial-wave capacity for fits that start at ``starts`` (B, 6): room
    for a_p to grow 25 % and n_p by 0.25 during the fit.'''
    a = starts[:, 3] * 1.25
    n = starts[:, 4] + 0.25
    k = starts[:, 5]
    return K.nmax_cap_for(a, n, k, n_m, wavelength, margin=4)


class PackedFeatures:
    '''Crops packed for the device: float32 data, lmb_feature records and
    optional float32 (x, y) coordinates for non-grid pixel sets.'''

    def __init__(self, items):
        '''items: list of (data (npix,) or (ny, nx), grid) where grid is
        (x0, y0, ny, nx) or None with explicit coords (2, npix).'''
        feats = np.zeros(len(items), dtype=_native.FEATURE_DTYPE)
        chunks, cchunks = [], []
        off = 0
        explicit = any(it[1] is None for it in items)
        for i, (data, grid, coords) in enumerate(items):
            d = np.ascontiguousarray(np.ravel(data), dtype=np.float32)
            n = d.size
            if grid is not None:
                x0, y0, ny, nx = grid
                if ny * nx != n:
                    raise ValueError('data size does not match its grid')
                feats[i] = (x0, y0, nx, ny, n, off)
            else:
                feats[i] = (0., 0., 0, 0, n, off)
            chunks.append(d)
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
        self.data = (np.concatenate(chunks) if chunks
                     else np.zeros(0, np.float32))
        self.coords = (np.concatenate(cchunks).reshape(-1)
                       if explicit and cchunks else None)
        self.total = off

    @property
    def h2d_bytes(self):
        n = self.data.nbytes + self.features.nbytes
        if self.coords is not None:
            n += self.coords.nbytes
        return n


def _to_device(a, dev):
    t = torch.from_numpy(np.ascontiguousarray(a))
    if t.numel() == 0:
        return t.to(dev)
    return t.pin_memory().to(dev, non_blocking=True)


def fit_packed(packed, starts, instrument, variables, settings=None,
               device=None, nmax_cap=None):
    '''Fit every packed feature; returns (params (B, 6), results record
    array with dparams, redchi, cost, status, success, nfev, njev).'''
    dev = get_device(device)
    lib = _native.load()
    settings = dict(DEFAULT_SETTINGS if settings is None else settings)
    starts = np.ascontiguousarray(starts, dtype=np.float64).reshape(-1, 6)
    B = starts.shape[0]
    res = np.zeros(B, dtype=_native.RESULT_DTYPE)
    if B == 0:
        return starts.copy(), res
    n_m = float(instrument.n_m)
    lam = float(instrument.wavelength)
    cap = nmax_cap or fit_capacity(starts, n_m, lam)
    d_data = _to_device(packed.data, dev)
    d_feat = _to_device(packed.features.view(np.uint8), dev)
    d_coords = (_to_device(packed.coords, dev) if packed.coords is not None
                else None)
    d_params = _to_device(starts, dev)
    d_res = torch.empty(B * _native.RESULT_DTYPE.itemsize, dtype=torch.uint8,
                        device=dev)
    nbytes = lib.lmb_fit_workspace_bytes(B, packed.total, cap)
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
    _native.check(lib.lmb_fit_batch(
        ptr(d_feat), B, packed.total, ptr(d_data), ptr(d_coords),
        ptr(d_params), n_m, lam, float(instrument.magnification),
        float(instrument.noise), cap, st, ptr(d_res), ptr(ws), nbytes,
        stream_handle(dev)), 'lmb_fit_batch')
    params = d_params.cpu().numpy()
    res = d_res.cpu().numpy().view(_native.RESULT_DTYPE).copy()
    return params, res
