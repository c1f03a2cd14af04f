'''Tensor-level wrappers of the C-ABI kernels (device memory via torch).

Every function takes and returns CUDA tensors, launches on torch's current
stream of the tensors' device, and raises ``LMBError`` on a non-zero
status.  Layouts are those of include/lmb200.h.
'''
import numpy as np
import torch

from .. import _native
from .._device import get_device, stream_handle, ptr

SPHERE_DTYPE = _native.SPHERE_DTYPE


def wiscombe_yang(a_p, n_p, k_p, n_m, wavelength):
    '''Host evaluation of Sphere.wiscombe_yang for arrays of spheres.'''
    k = 2. * np.pi / wavelength * float(np.real(n_m))
    x = np.abs(k * np.asarray(a_p, dtype=float))
    m = (np.asarray(n_p, dtype=float) + 1j * np.asarray(k_p, dtype=float)) / n_m
    ns = np.where(x <= 8., np.floor(x + 4. * np.cbrt(x) + 1.),
                  np.where(x <= 4200., np.floor(x + 4.05 * np.cbrt(x) + 2.),
                           np.floor(x + 4. * np.cbrt(x) + 2.)))
    return np.maximum(ns, np.abs(x * m)).astype(np.int64)


def nmax_cap_for(a_p, n_p, k_p, n_m, wavelength, margin=2):
    '''Order capacity covering these spheres (small margin for rounding).'''
    nm = wiscombe_yang(a_p, n_p, k_p, n_m, wavelength)
    cap = int(nm.max()) + margin if nm.size else 1
    if cap > _native.LMB_NMAX_LIMIT:
        raise ValueError(f'sphere needs {int(nm.max())} partial-wave orders; '
                         f'the limit is {_native.LMB_NMAX_LIMIT}')
    return max(cap, 1)


def spheres_tensor(records, device):
    '''(n, 6) float64 device tensor from a SPHERE_DTYPE array.'''
    a = np.ascontiguousarray(records).view(np.float64).reshape(-1, 6)
    return torch.from_numpy(a.copy()).to(device, non_blocking=False)


def sphere_ab(spheres, n_m, wavelength, cap, deriv=False, check=True):
    '''Mie coefficients of (n, 6) spheres: ab (n, cap+1, 2, 2) float64
    (complex interleaved), dab (n, cap+1, 4, 2) or None, nmax (n,) int32.'''
    lib = _native.load()
    dev = spheres.device
    n = spheres.shape[0]
    ab = torch.empty((n, cap + 1, 2, 2), dtype=torch.float64, device=dev)
    dab = (torch.empty((n, cap + 1, 4, 2), dtype=torch.float64, device=dev)
           if deriv else None)
    nmax = torch.empty(n, dtype=torch.int32, device=dev)
    status = torch.empty(n, dtype=torch.int32, device=dev)
    _native.check(lib.lmb_sphere_ab(ptr(spheres), n, float(n_m),
                                    float(wavelength), cap, ptr(ab), ptr(dab),
                                    ptr(nmax), ptr(status),
                                    stream_handle(dev)), 'lmb_sphere_ab')
    if check and n and int(status.max().item()) != _native.LMB_OK:
        raise ValueError('a sphere needs more partial-wave orders than the '
                         f'capacity {cap}')
    return ab, dab, nmax


def sphere_ab_host(records, n_m, wavelength, deriv=False):
    '''Coefficients for host sphere records, returned as numpy complex.'''
    dev = get_device()
    cap = nmax_cap_for(records['a_p'], records['n_p'], records['k_p'], n_m,
                       wavelength)
    sp = spheres_tensor(records, dev)
    ab, dab, nmax = sphere_ab(sp, n_m, wavelength, cap, deriv)
    a = ab.cpu().numpy()
    a = a[..., 0] + 1j * a[..., 1]
    d = None
    if deriv:
        d = dab.cpu().numpy()
        d = d[..., 0] + 1j * d[..., 1]
    return a, d, nmax.cpu().numpy()


def _flags(cartesian, bohren, fp64):
    return ((_native.LMB_CARTESIAN if cartesian else 0) |
            (_native.LMB_BOHREN if bohren else 0) |
            (_native.LMB_FP64 if fp64 else 0))


def hologram(coords, spheres, item_start, ab, nmax, cap, k, cartesian=True,
             bohren=True, fp64=False):
    '''(nitems, npts) holograms; float32, or float64 when fp64.'''
    lib = _native.load()
    dev = coords.device
    npts = coords.shape[1]
    nitems = item_start.shape[0] - 1
    out = torch.empty((nitems, npts),
                      dtype=torch.float64 if fp64 else torch.float32,
                      device=dev)
    _native.check(lib.lmb_hologram(ptr(coords), npts, ptr(spheres),
                                   ptr(item_start), nitems, ptr(ab), ptr(nmax),
                                   cap, float(k),
                                   _flags(cartesian, bohren, fp64), ptr(out),
                                   stream_handle(dev)), 'lmb_hologram')
    return out


def field(coords, spheres, item_start, ab, nmax, cap, k, cartesian=True,
          bohren=True, fp64=False):
    '''(nitems, 3, npts) scattered fields; complex64, or complex128.'''
    lib = _native.load()
    dev = coords.device
    npts = coords.shape[1]
    nitems = item_start.shape[0] - 1
    out = torch.empty((nitems, 3, npts),
                      dtype=torch.complex128 if fp64 else torch.complex64,
                      device=dev)
    _native.check(lib.lmb_field(ptr(coords), npts, ptr(spheres),
                                ptr(item_start), nitems, ptr(ab), ptr(nmax),
                                cap, float(k), _flags(cartesian, bohren, fp64),
                                ptr(out), stream_handle(dev)), 'lmb_field')
    return out


def jacobian(coords, spheres, ab, dab, nmax, cap, k, bohren=True):
    '''Holograms (n, npts) and Jacobians (n, 6, npts), float64, FP32 sums.'''
    lib = _native.load()
    dev = coords.device
    npts = coords.shape[1]
    n = spheres.shape[0]
    holo = torch.empty((n, npts), dtype=torch.float64, device=dev)
    jac = torch.empty((n, 6, npts), dtype=torch.float64, device=dev)
    _native.check(lib.lmb_jacobian(ptr(coords), npts, ptr(spheres), n, ptr(ab),
                                   ptr(dab), ptr(nmax), cap, float(k),
                                   _flags(True, bohren, False), ptr(holo),
                                   ptr(jac), stream_handle(dev)),
                  'lmb_jacobian')
    return holo, jac


def hologram_vjp(coords, spheres, ab, dab, nmax, cap, k, gout, bohren=True):
    '''sum_p gout[i, p] dH_i[p]/dparam_j -> (n, 6) float64.'''
    lib = _native.load()
    dev = coords.device
    npts = coords.shape[1]
    n = spheres.shape[0]
    gout = gout.to(torch.float32).contiguous()
    grad = torch.empty((n, 6), dtype=torch.float64, device=dev)
    nbytes = lib.lmb_vjp_workspace_bytes(npts, n)
    ws = torch.empty(max(nbytes, 1), dtype=torch.uint8, device=dev)
    _native.check(lib.lmb_hologram_vjp(ptr(coords), npts, ptr(spheres), n,
                                       ptr(ab), ptr(dab), ptr(nmax), cap,
                                       float(k), _flags(True, bohren, False),
                                       ptr(gout), ptr(grad), ptr(ws), nbytes,
                                       stream_handle(dev)),
                  'lmb_hologram_vjp')
    return grad
