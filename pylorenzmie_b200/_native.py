'''ctypes binding of the in-tree CUDA library ``_lib/liblmb200.so``.

The library's C ABI is declared in ``include/lmb200.h``.  This module loads
the in-tree build (building it first when the sources are newer and nvcc
is available) and fails loudly otherwise: there is no CPU fallback.
'''
import ctypes
import threading

import numpy as np

from . import build as _build

LMB_OK = 0
LMB_ERR_ARG = 1
LMB_ERR_CUDA = 2
LMB_ERR_NMAX = 3
LMB_ERR_WORKSPACE = 4
LMB_ERR_UNSUPPORTED = 5
LMB_ERR_TIMEOUT = 6
LMB_PACK_F64 = 0
LMB_PACK_F32 = 1

LMB_CARTESIAN = 1
LMB_BOHREN = 2
LMB_FP64 = 4
LMB_NMAX_LIMIT = 1024

# struct layouts mirrored from include/lmb200.h
SPHERE_DTYPE = np.dtype([('x_p', '<f8'), ('y_p', '<f8'), ('z_p', '<f8'),
                         ('a_p', '<f8'), ('n_p', '<f8'), ('k_p', '<f8')])
FEATURE_DTYPE = np.dtype([('x0', '<f8'), ('y0', '<f8'), ('nx', '<i4'),
                          ('ny', '<i4'), ('npix', '<i8'),
                          ('data_offset', '<i8')])
RESULT_DTYPE = np.dtype([('dparams', '<f8', (6,)), ('redchi', '<f8'),
                         ('cost', '<f8'), ('status', '<i4'),
                         ('success', '<i4'), ('nfev', '<i4'),
                         ('njev', '<i4')])


class FitSettings(ctypes.Structure):
    _fields_ = [('ftol', ctypes.c_double), ('xtol', ctypes.c_double),
                ('gtol', ctypes.c_double), ('factor', ctypes.c_double),
                ('max_nfev', ctypes.c_int), ('variables', ctypes.c_int),
                ('flags', ctypes.c_int), ('max_iterations', ctypes.c_int),
                ('tile_config', ctypes.c_int), ('reserved', ctypes.c_int)]


class FitStats(ctypes.Structure):
    _fields_ = [('eval_ms', ctypes.c_double), ('total_ms', ctypes.c_double),
                ('pixels', ctypes.c_double), ('pixel_orders', ctypes.c_double),
                ('eval_launches', ctypes.c_int),
                ('kernel_launches', ctypes.c_int),
                ('iterations', ctypes.c_int), ('pad', ctypes.c_int)]


class LMBError(RuntimeError):
    '''A non-zero status from the CUDA library.'''

    def __init__(self, status, where):
        self.status = status
        super().__init__(f'{where}: {status_string(status)} (status {status})')


_vp = ctypes.c_void_p
_ll = ctypes.c_longlong
_i = ctypes.c_int
_d = ctypes.c_double
_sz = ctypes.c_size_t

_SIGNATURES = {
    'lmb_version': (_i, []),
    'lmb_status_string': (ctypes.c_char_p, [_i]),
    'lmb_sphere_ab': (_i, [_vp, _i, _d, _d, _i, _vp, _vp, _vp, _vp, _vp]),
    'lmb_layered_ab': (_i, [_vp, _vp, _i, _i, _d, _d, _i, _vp, _vp, _vp,
                            _vp, _vp]),
    'lmb_field': (_i, [_vp, _ll, _vp, _vp, _i, _vp, _vp, _i, _d, _i, _vp,
                       _vp]),
    'lmb_hologram': (_i, [_vp, _ll, _vp, _vp, _i, _vp, _vp, _i, _d, _i, _vp,
                          _vp]),
    'lmb_field_aberrated': (_i, [_vp, _ll, _vp, _vp, _i, _vp, _vp, _i, _d,
                                 _i, _d, _vp, _vp]),
    'lmb_hologram_aberrated': (_i, [_vp, _ll, _vp, _vp, _i, _vp, _vp, _i,
                                    _d, _i, _d, _vp, _vp]),
    'lmb_jacobian': (_i, [_vp, _ll, _vp, _i, _vp, _vp, _vp, _i, _d, _i, _vp,
                          _vp, _vp]),
    'lmb_de_trial': (_i, [_i, _i, _vp, _i, _i, _vp, _vp, _vp, _i, _d, _d,
                          _vp, _vp, _vp, _vp, _vp, _vp, _i, _vp, _vp]),
    'lmb_de_select': (_i, [_i, _i, _vp, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp,
                           _vp, _vp, _vp, _i, _vp]),
    'lmb_jacobian_aberrated': (_i, [_vp, _ll, _vp, _i, _vp, _vp, _vp, _i, _d,
                                    _i, _d, _vp, _vp, _vp]),
    'lmb_vjp_workspace_bytes': (_sz, [_ll, _i]),
    'lmb_hologram_vjp': (_i, [_vp, _ll, _vp, _i, _vp, _vp, _vp, _i, _d, _i,
                              _vp, _vp, _vp, _sz, _vp]),
    'lmb_fit_workspace_bytes': (_sz, [_i, _ll, _i]),
    'lmb_chi2_workspace_bytes': (_sz, [_ll, _i]),
    'lmb_chi2_batch': (_i, [_vp, _ll, _vp, _d, _vp, _vp, _i, _vp, _vp, _i,
                            _d, _i, _vp, _vp, _vp, _sz, _vp]),
    'lmb_chi2_crops': (_i, [_vp, _ll, _vp, _d, _vp, _i, _vp, _ll, _vp, _vp,
                            _i, _vp, _vp, _i, _d, _i, _vp, _vp, _vp, _sz,
                            _vp, _d]),
    'lmb_fit_batch_layered': (_i, [_vp, _i, _ll, _vp, _vp, _vp, _i, _vp, _vp,
                                   _d, _d, _d, _d, _i,
                                   ctypes.POINTER(FitSettings), _vp, _vp, _sz,
                                   ctypes.POINTER(FitStats), _vp]),
    'lmb_fit_batch_aberrated': (_i, [_vp, _i, _ll, _vp, _vp, _vp, _i, _vp,
                                     _vp, _d, _d, _d, _d, _i, _d,
                                     ctypes.POINTER(FitSettings), _vp, _vp,
                                     _sz, ctypes.POINTER(FitStats), _vp]),
    'lmb_fit_batch_streamed': (_i, [_vp, _i, _ll, _vp, _vp, _vp, _i, _vp,
                                    _vp, _d, _d, _d, _d, _i,
                                    ctypes.POINTER(FitSettings), _vp, _d,
                                    _vp, _vp, _sz, ctypes.POINTER(FitStats),
                                    _vp, _d]),
    'lmb_fit_tile_config': (_i, [_i, ctypes.POINTER(_i), ctypes.POINTER(_i),
                                 ctypes.POINTER(_i)]),
    'lmb_fit_batch': (_i, [_vp, _i, _ll, _vp, _vp, _vp, _d, _d, _d, _d, _i,
                           ctypes.POINTER(FitSettings), _vp, _vp, _sz,
                           ctypes.POINTER(FitStats), _vp]),
    'lmb_measure_fp32_peak': (_i, [ctypes.POINTER(_d), _vp]),
    'lmb_pack_crops': (_i, [_vp, _vp, _i, _i, _vp, _i]),
    'lmb_de_shuffles': (_i, [_vp, _vp, _ll, _ll, _i, _vp]),
    'lmb_de_draws': (_i, [_vp, _i, _i, _d, _d, _vp, _vp, _ll, _i, _vp, _i,
                          _d, _vp, _vp]),
    'lmb_mask_select': (_i, [_vp, _ll, _d, _vp, _i, _vp, _vp]),
    'lmb_de_draws_many': (_i, [_i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _ll,
                               _i, _vp, _i, _vp, _vp, _vp]),
}

_lock = threading.Lock()
_lib = None


def library_path():
    return _build.LIBRARY


def load():
    '''Load (building if stale) the CUDA library; raise if impossible.'''
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        path = _build.LIBRARY
        if not _build.up_to_date():
            try:
                path = _build.build()
            except Exception as e:  # no nvcc here: use what is on disk
                if not path.exists():
                    raise ImportError(
                        'pylorenzmie_b200 CUDA library is missing and could '
                        f'not be built: {e}') from e
        lib = ctypes.CDLL(str(path))
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def status_string(status):
    try:
        return load().lmb_status_string(int(status)).decode()
    except Exception:
        return 'unknown status'


def check(status, where):
    if status != LMB_OK:
        raise LMBError(status, where)


def symbols():
    '''Names of the C entry points this binding expects.'''
    return list(_SIGNATURES)
