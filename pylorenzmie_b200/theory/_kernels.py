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


def to_device_async(array, device):
    '''Device copy of a small host array through pinned memory, queued on
    the current stream without waiting for the work already queued there
    (a pageable copy would wait for it).'''
    host = torch.from_numpy(np.ascontiguousarray(array).copy())
    if torch.cuda.is_available():
        host = host.pin_memory()
    return host.to(device, non_blocking=True)


def to_numpy(tensor, dtype):
    '''A device tensor as a new numpy array of torch ``dtype``: converted
    on the device, then copied in one DMA into page-locked host memory from
    torch's caching host allocator and handed to numpy without a further
    copy.  A copy into pageable memory goes through a staging buffer at a
    fraction of the link's speed (41 MB of holograms: 19 ms against 3.5 ms
    on a B200 host).  Small tensors take the plain copy.'''
    t = tensor.to(dtype)
    if t.device.type != 'cuda' or t.numel() * t.element_size() < (1 << 18):
        return t.cpu().numpy()
    out = torch.empty(t.shape, dtype=dtype, pin_memory=True)
    with torch.cuda.device(t.device):
        out.copy_(t, non_blocking=True)
        torch.cuda.current_stream().synchronize()
    return out.numpy()


def spheres_tensor(records, device):
    '''(n, 6) float64 device tensor from a SPHERE_DTYPE array.'''
    a = np.ascontiguousarray(records).view(np.float64).reshape(-1, 6)
    return to_device_async(a, device)


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


def _contiguous(*tensors):
    '''Row-major copies where needed: the library reads plain pointers.'''
    return tuple(None if t is None else t.contiguous() for t in tensors)


def _flags(cartesian, bohren, fp64):
    return ((_native.LMB_CARTESIAN if cartesian else 0) |
            (_native.LMB_BOHREN if bohren else 0) |
            (_native.LMB_FP64 if fp64 else 0))


def hologram(coords, spheres, item_start, ab, nmax, cap, k, cartesian=True,
             bohren=True, fp64=False, aberration=0.):
    '''(nitems, npts) holograms; float32, or float64 when fp64.
    ``aberration``: coefficient 4 n_m^3 s / k of a spherical-aberration
    phase (0: none).'''
    coords, spheres, item_start, ab, nmax = _contiguous(
        coords, spheres, item_start, ab, nmax)
    lib = _native.load()
    dev = coords.device
    npts = coords.shape[1]
    nitems = item_start.shape[0] - 1
    out = torch.empty((nitems, npts),
                      dtype=torch.float64 if fp64 else torch.float32,
                      device=dev)
    flags = _flags(cartesian, bohren, fp64)
    if aberration:
        _native.check(lib.lmb_hologram_aberrated(
            ptr(coords), npts, ptr(spheres), ptr(item_start), nitems, ptr(ab),
            ptr(nmax), cap, float(k), flags, float(aberration), ptr(out),
            stream_handle(dev)), 'lmb_hologram_aberrated')
        return out
    _native.check(lib.lmb_hologram(ptr(coords), npts, ptr(spheres),
                                   ptr(item_start), nitems, ptr(ab), ptr(nmax),
                                   cap, float(k), flags, ptr(out),
                                   stream_handle(dev)), 'lmb_hologram')
    return out


def chi2(coords, data, noise, spheres, item_start, ab, nmax, cap, k,
         cartesian=True, bohren=True, fp64=False, nonfinite=False):
    '''(nitems,) float64 sums of ((hologram - data) / noise)^2, NaN
    residuals skipped (lmb_chi2_batch); with ``nonfinite`` also the
    (nitems,) int32 counts of NaN or infinite hologram pixels.'''
    coords, data, spheres, item_start, ab, nmax = _contiguous(
        coords, data, spheres, item_start, ab, nmax)
    lib = _native.load()
    dev = coords.device
    npts = coords.shape[1]
    nitems = item_start.shape[0] - 1
    out = torch.empty(max(nitems, 1), dtype=torch.float64, device=dev)
    bad = torch.empty(max(nitems, 1), dtype=torch.int32, device=dev) \
        if nonfinite else None
    nbytes = lib.lmb_chi2_workspace_bytes(npts, nitems)
    ws = torch.empty(max(nbytes, 1), dtype=torch.uint8, device=dev)
    _native.check(lib.lmb_chi2_batch(ptr(coords), npts, ptr(data),
                                     float(noise), ptr(spheres),
                                     ptr(item_start), nitems, ptr(ab),
                                     ptr(nmax), cap, float(k),
                                     _flags(cartesian, bohren, fp64),
                                     ptr(out), ptr(bad), ptr(ws), nbytes,
                                     stream_handle(dev)), 'lmb_chi2_batch')
    if nonfinite:
        return out[:nitems], bad[:nitems]
    return out[:nitems]


def chi2_crops(coords, data, noise, crop_start, item_crop, max_crop_npts,
               spheres, item_start, ab, nmax, cap, k, cartesian=True,
               bohren=True, fp64=False, aberration=0.):
    '''chi2 as above with item i compared with the pixels of its own crop
    item_crop[i], [crop_start[c], crop_start[c + 1]) of coords and data
    (lmb_chi2_crops): (nitems,) float64 sums and (nitems,) int32 counts of
    NaN or infinite hologram pixels.  ``aberration``: the coefficient c of
    the spherical-aberration phase (0: ideal optics).'''
    coords, data, crop_start, item_crop, spheres, item_start, ab, nmax = \
        _contiguous(coords, data, crop_start, item_crop, spheres, item_start,
                    ab, nmax)
    lib = _native.load()
    dev = coords.device
    npts = coords.shape[1]
    nitems = item_start.shape[0] - 1
    ncrops = crop_start.shape[0] - 1
    out = torch.empty(max(nitems, 1), dtype=torch.float64, device=dev)
    bad = torch.empty(max(nitems, 1), dtype=torch.int32, device=dev)
    nbytes = lib.lmb_chi2_workspace_bytes(int(max_crop_npts), nitems)
    ws = torch.empty(max(nbytes, 1), dtype=torch.uint8, device=dev)
    _native.check(lib.lmb_chi2_crops(
        ptr(coords), npts, ptr(data), float(noise), ptr(crop_start), ncrops,
        ptr(item_crop), int(max_crop_npts), ptr(spheres), ptr(item_start),
        nitems, ptr(ab), ptr(nmax), cap, float(k),
        _flags(cartesian, bohren, fp64), ptr(out), ptr(bad), ptr(ws), nbytes,
        stream_handle(dev), float(aberration)), 'lmb_chi2_crops')
    return out[:nitems], bad[:nitems]


def field(coords, spheres, item_start, ab, nmax, cap, k, cartesian=True,
          bohren=True, fp64=False, aberration=0.):
    '''(nitems, 3, npts) scattered fields; complex64, or complex128.'''
    coords, spheres, item_start, ab, nmax = _contiguous(
        coords, spheres, item_start, ab, nmax)
    lib = _native.load()
    dev = coords.device
    npts = coords.shape[1]
    nitems = item_start.shape[0] - 1
    out = torch.empty((nitems, 3, npts),
                      dtype=torch.complex128 if fp64 else torch.complex64,
                      device=dev)
    flags = _flags(cartesian, bohren, fp64)
    if aberration:
        _native.check(lib.lmb_field_aberrated(
            ptr(coords), npts, ptr(spheres), ptr(item_start), nitems, ptr(ab),
            ptr(nmax), cap, float(k), flags, float(aberration), ptr(out),
            stream_handle(dev)), 'lmb_field_aberrated')
        return out
    _native.check(lib.lmb_field(ptr(coords), npts, ptr(spheres),
                                ptr(item_start), nitems, ptr(ab), ptr(nmax),
                                cap, float(k), flags, ptr(out),
                                stream_handle(dev)), 'lmb_field')
    return out


def jacobian(coords, spheres, ab, dab, nmax, cap, k, bohren=True,
             aberration=0.):
    '''Holograms (n, npts) and Jacobians (n, 6, npts), float64, FP32 sums;
    ``aberration``: the coefficient c of the spherical-aberration phase
    (lmb_jacobian_aberrated; 0: ideal optics).'''
    coords, spheres, ab, dab, nmax = _contiguous(
        coords, spheres, ab, dab, nmax)
    lib = _native.load()
    dev = coords.device
    npts = coords.shape[1]
    n = spheres.shape[0]
    holo = torch.empty((n, npts), dtype=torch.float64, device=dev)
    jac = torch.empty((n, 6, npts), dtype=torch.float64, device=dev)
    if aberration:
        _native.check(lib.lmb_jacobian_aberrated(
            ptr(coords), npts, ptr(spheres), n, ptr(ab), ptr(dab), ptr(nmax),
            cap, float(k), _flags(True, bohren, False), float(aberration),
            ptr(holo), ptr(jac), stream_handle(dev)), 'lmb_jacobian_aberrated')
        return holo, jac
    _native.check(lib.lmb_jacobian(ptr(coords), npts, ptr(spheres), n, ptr(ab),
                                   ptr(dab), ptr(nmax), cap, float(k),
                                   _flags(True, bohren, False), ptr(holo),
                                   ptr(jac), stream_handle(dev)),
                  'lmb_jacobian')
    return holo, jac


def hologram_vjp(coords, spheres, ab, dab, nmax, cap, k, gout, bohren=True):
    '''sum_p gout[i, p] dH_i[p]/dparam_j -> (n, 6) float64.'''
    coords, spheres, ab, dab, nmax, gout = _contiguous(
        coords, spheres, ab, dab, nmax, gout)
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


def wiscombe_yang_layers(radii, indices, n_m, wavelength):
    '''Host n_max of one multilayer sphere (radii ascending, complex indices).'''
    k = 2. * np.pi / wavelength * float(np.real(n_m))
    x = k * np.asarray(radii, dtype=float)
    m = np.asarray(indices, dtype=complex) / n_m
    xl = abs(x[-1])
    if xl <= 8.:
        ns = np.floor(xl + 4. * np.cbrt(xl) + 1.)
    elif xl <= 4200.:
        ns = np.floor(xl + 4.05 * np.cbrt(xl) + 2.)
    else:
        ns = np.floor(xl + 4. * np.cbrt(xl) + 2.)
    return int(max(ns, np.abs(x * m).max(), np.abs(np.roll(x, -1) * m).max()))


def layered_ab(radii, indices, n_m, wavelength, cap, deriv=False, check=True):
    '''Coefficients of multilayer spheres: radii (n, L), indices (n, L, 2)
    float64 device tensors; outputs as sphere_ab.'''
    lib = _native.load()
    dev = radii.device
    n, L = radii.shape
    ab = torch.empty((n, cap + 1, 2, 2), dtype=torch.float64, device=dev)
    dab = (torch.empty((n, cap + 1, 4, 2), dtype=torch.float64, device=dev)
           if deriv else None)
    nmax = torch.empty(n, dtype=torch.int32, device=dev)
    status = torch.empty(n, dtype=torch.int32, device=dev)
    _native.check(lib.lmb_layered_ab(ptr(radii), ptr(indices), L, n,
                                     float(n_m), float(wavelength), cap,
                                     ptr(ab), ptr(dab), ptr(nmax),
                                     ptr(status), stream_handle(dev)),
                  'lmb_layered_ab')
    if check and n and int(status.max().item()) != _native.LMB_OK:
        raise ValueError('a layered sphere is invalid or needs more '
                         f'partial-wave orders than the capacity {cap}')
    return ab, dab, nmax


def is_layered(p):
    return hasattr(p, 'fractions') and hasattr(p, 'core_indices')


def particle_nmax(p, n_m, wavelength):
    if is_layered(p):
        return wiscombe_yang_layers(p.radii, p.indices, n_m, wavelength)
    return int(wiscombe_yang(p.a_p, p.n_p, getattr(p, 'k_p', 0.), n_m,
                             wavelength))


def particle_ab(particles, spheres, n_m, wavelength, cap, deriv=False,
                check=True):
    '''Coefficients for a list of Sphere / LayeredSphere particles (in
    order); spheres is their (n, 6) device tensor.  ``check=False`` skips
    the status read-back (a device round trip) for homogeneous spheres
    whose parameters the caller has validated.'''
    dev = spheres.device
    n = len(particles)
    layered = [i for i, p in enumerate(particles) if is_layered(p)]
    if not layered:
        return sphere_ab(spheres, n_m, wavelength, cap, deriv, check=check)
    ab = torch.zeros((n, cap + 1, 2, 2), dtype=torch.float64, device=dev)
    dab = (torch.zeros((n, cap + 1, 4, 2), dtype=torch.float64, device=dev)
           if deriv else None)
    nmax = torch.zeros(n, dtype=torch.int32, device=dev)
    plain = [i for i in range(n) if i not in set(layered)]
    if plain:
        idx = torch.tensor(plain, device=dev)
        a, d, m = sphere_ab(spheres[idx].contiguous(), n_m, wavelength, cap,
                            deriv)
        ab[idx], nmax[idx] = a, m
        if deriv:
            dab[idx] = d
    groups = {}
    for i in layered:
        groups.setdefault(particles[i].nlayers, []).append(i)
    for L, members in groups.items():
        r = np.array([particles[i].radii for i in members], dtype=float)
        ind = np.zeros((len(members), L, 2))
        for j, i in enumerate(members):
            ind[j, :, 0] = particles[i].indices.real
            ind[j, :, 1] = particles[i].indices.imag
        a, d, m = layered_ab(torch.from_numpy(r).to(dev),
                             torch.from_numpy(ind).to(dev), n_m, wavelength,
                             cap, deriv)
        idx = torch.tensor(members, device=dev)
        ab[idx], nmax[idx] = a, m
        if deriv:
            dab[idx] = d
    return ab, dab, nmax


def layered_ab_host(particles, n_m, wavelength, deriv=False):
    '''Coefficients of LayeredSphere particles as numpy complex arrays.'''
    dev = get_device()
    cap = max(particle_nmax(p, n_m, wavelength) for p in particles) + 2
    rec = np.zeros(len(particles), dtype=SPHERE_DTYPE)
    for i, p in enumerate(particles):
        rec[i] = (0., 0., 0., p.a_p, p.n_p, p.k_p)
    ab, dab, nmax = particle_ab(particles, spheres_tensor(rec, dev), n_m,
                                wavelength, cap, deriv)
    a = ab.cpu().numpy()
    a = a[..., 0] + 1j * a[..., 1]
    d = None
    if deriv:
        d = dab.cpu().numpy()
        d = d[..., 0] + 1j * d[..., 1]
    return a, d, nmax.cpu().numpy()
