'''Compile and load the CPU harness (tests only).'''
import ctypes
import shutil
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
CSRC = ROOT / 'pylorenzmie_b200' / 'csrc'
BUILD = HERE / '_build'
LIB = BUILD / 'libharness.so'

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def _stale():
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    srcs = [HERE / 'harness.cpp', *CSRC.glob('*.cuh')]
    return any(s.stat().st_mtime > t for s in srcs)


def load():
    if _stale():
        cxx = shutil.which('g++') or shutil.which('c++')
        if cxx is None:
            raise RuntimeError('no C++ compiler for the CPU harness')
        BUILD.mkdir(exist_ok=True)
        tmp = LIB.with_suffix('.tmp')
        subprocess.run([cxx, '-O2', '-shared', '-fPIC', '-std=c++17',
                        f'-I{CSRC}', str(HERE / 'harness.cpp'), '-o',
                        str(tmp)], check=True)
        tmp.replace(LIB)
    lib = ctypes.CDLL(str(LIB))
    lib.h_sphere_ab.argtypes = [ctypes.c_double] * 5 + [ctypes.c_int, _dp, _dp, _ip]
    lib.h_layered_ab.argtypes = [_dp, _dp, ctypes.c_int, ctypes.c_double,
                                 ctypes.c_double, ctypes.c_int, _dp, _dp, _ip]
    lib.h_layered_ab_split.argtypes = lib.h_layered_ab.argtypes
    lib.h_field.argtypes = [_dp, ctypes.c_longlong, _dp, _dp, ctypes.c_int,
                            ctypes.c_double, ctypes.c_int, ctypes.c_int, _dp]
    lib.h_jacobian.argtypes = [_dp, ctypes.c_longlong, _dp, _dp, _dp,
                               ctypes.c_int, ctypes.c_double, ctypes.c_int,
                               ctypes.c_int, _dp, _dp]
    lib.h_jacobian_rev.argtypes = [_dp, ctypes.c_longlong, _dp, _dp, _dp,
                                   ctypes.c_int, ctypes.c_double,
                                   ctypes.c_int, ctypes.c_int, _dp, _dp]
    lib.h_jacobian_aberrated.argtypes = [_dp, ctypes.c_longlong, _dp, _dp,
                                         _dp, ctypes.c_int, ctypes.c_double,
                                         ctypes.c_int, ctypes.c_int,
                                         ctypes.c_double, _dp, _dp]
    lib.h_field_pair.argtypes = [_dp, ctypes.c_longlong, _dp, _dp,
                                 ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                 _dp]
    lib.h_hologram_pair.argtypes = [_dp, ctypes.c_longlong, _dp, ctypes.c_int,
                                    _dp, _ip, ctypes.c_int, ctypes.c_double,
                                    ctypes.c_int,
                                    ctypes.POINTER(ctypes.c_float),
                                    ctypes.POINTER(ctypes.c_float)]
    lib.h_jacobian_pair.argtypes = [_dp, ctypes.c_longlong, _dp, _dp, _dp,
                                    ctypes.c_int, ctypes.c_double,
                                    ctypes.c_int, _dp, _dp]
    lib.h_lm_new.restype = ctypes.c_void_p
    lib.h_lm_new.argtypes = [ctypes.c_int, _ip, _dp] + [ctypes.c_double] * 4 + [ctypes.c_int]
    lib.h_lm_free.argtypes = [ctypes.c_void_p]
    lib.h_lm_feed.argtypes = [ctypes.c_void_p, ctypes.c_double, _dp, _dp, _dp]
    lib.h_lm_result.argtypes = [ctypes.c_void_p, ctypes.c_longlong, _dp, _ip,
                                _ip, _ip, _dp, _dp]
    return lib


def ptr(a, t=_dp):
    return a.ctypes.data_as(t)


class Harness:
    '''Thin numpy wrappers around the harness entry points.'''

    def __init__(self):
        self.lib = load()

    def sphere_ab(self, a_p, n_p, k_p, n_m, wavelength, cap=1024, deriv=False):
        ab = np.zeros((cap + 1, 2, 2))
        dab = np.zeros((cap + 1, 4, 2)) if deriv else None
        nmax = ctypes.c_int()
        st = self.lib.h_sphere_ab(a_p, n_p, k_p, n_m, wavelength, cap, ptr(ab),
                                  ptr(dab) if deriv else None,
                                  ctypes.byref(nmax))
        if st != 0:
            raise ValueError(f'nmax {nmax.value} above cap')
        n = nmax.value
        ab = ab[:n + 1, :, 0] + 1j * ab[:n + 1, :, 1]
        if deriv:
            dab = dab[:n + 1, :, 0] + 1j * dab[:n + 1, :, 1]
            return ab, dab
        return ab

    def layered_ab(self, radii, indices, n_m, wavelength, cap=1024,
                   deriv=False, split=False):
        r = np.ascontiguousarray(radii, dtype=float)
        idx = np.zeros((r.size, 2))
        idx[:, 0] = np.real(indices)
        idx[:, 1] = np.imag(indices)
        ab = np.zeros((cap + 1, 2, 2))
        dab = np.zeros((cap + 1, 4, 2)) if deriv else None
        nmax = ctypes.c_int()
        fn = self.lib.h_layered_ab_split if split else self.lib.h_layered_ab
        st = fn(ptr(r), ptr(idx), r.size, n_m, wavelength, cap, ptr(ab),
                ptr(dab) if deriv else None, ctypes.byref(nmax))
        if st != 0:
            raise ValueError(f'nmax {nmax.value} above cap')
        n = nmax.value
        ab = ab[:n + 1, :, 0] + 1j * ab[:n + 1, :, 1]
        if deriv:
            dab = dab[:n + 1, :, 0] + 1j * dab[:n + 1, :, 1]
            return ab, dab
        return ab

    @staticmethod
    def _pack_ab(ab, dab=None):
        n = ab.shape[0] - 1
        a = np.zeros((n + 1, 2, 2))
        a[..., 0] = ab.real
        a[..., 1] = ab.imag
        d = None
        if dab is not None:
            d = np.zeros((n + 1, 4, 2))
            d[..., 0] = dab.real
            d[..., 1] = dab.imag
        return n, a, d

    def field(self, coords, p, ab, k, cartesian=True, bohren=True, fp64=False):
        c = np.ascontiguousarray(coords, dtype=float)
        npts = c.shape[1]
        n, a, _ = self._pack_ab(ab)
        out = np.zeros((3, npts, 2))
        pv = np.asarray(p, dtype=float)
        flags = (1 if cartesian else 0) | (2 if bohren else 0)
        self.lib.h_field(ptr(c), npts, ptr(pv), ptr(a), n, k, flags, int(fp64),
                         ptr(out))
        return out[..., 0] + 1j * out[..., 1]

    def jacobian(self, coords, p, ab, dab, k, bohren=True, fp64=False):
        c = np.ascontiguousarray(coords, dtype=float)
        npts = c.shape[1]
        n, a, d = self._pack_ab(ab, dab)
        holo = np.zeros(npts)
        jac = np.zeros((6, npts))
        pv = np.asarray(p, dtype=float)
        self.lib.h_jacobian(ptr(c), npts, ptr(pv), ptr(a), ptr(d), n, k,
                            1 | (2 if bohren else 0), int(fp64), ptr(holo),
                            ptr(jac))
        return holo, jac

    def jacobian_pair(self, coords, p, ab, dab, k, bohren=True):
        '''As jacobian (FP32), through the packed two-pixel order loop.'''
        c = np.ascontiguousarray(coords, dtype=float)
        npts = c.shape[1]
        n, a, d = self._pack_ab(ab, dab)
        holo = np.zeros(npts)
        jac = np.zeros((6, npts))
        pv = np.asarray(p, dtype=float)
        self.lib.h_jacobian_pair(ptr(c), npts, ptr(pv), ptr(a), ptr(d), n, k,
                                 1 | (2 if bohren else 0), ptr(holo),
                                 ptr(jac))
        return holo, jac

    def field_pair(self, coords, p, ab, k, cartesian=True, bohren=True):
        '''(3, npts) complex field of one sphere through the packed
        two-pixel value loop (FP32).'''
        c = np.ascontiguousarray(coords, dtype=float)
        npts = c.shape[1]
        n, a, _ = self._pack_ab(ab)
        out = np.zeros((3, npts, 2))
        pv = np.asarray(p, dtype=float)
        self.lib.h_field_pair(ptr(c), npts, ptr(pv), ptr(a), n, k,
                              (1 if cartesian else 0) | (2 if bohren else 0),
                              ptr(out))
        return out[..., 0] + 1j * out[..., 1]

    def hologram_pair(self, coords, particles, k, cap=400, flag=True):
        '''FP32 hologram of several spheres (rows of x, y, z, a_p, n_p, k_p)
        as k_field_pair computes it: (H with -1 where its error bound asks
        for the FP64 sum (unless flag is False), the bound's two terms
        (2, npts)).'''
        c = np.ascontiguousarray(coords, dtype=float)
        npts = c.shape[1]
        P = np.ascontiguousarray(particles, dtype=float).reshape(-1, 6)
        ab = np.zeros((P.shape[0], cap + 1, 2, 2))
        nmax = np.zeros(P.shape[0], np.int32)
        for j, p in enumerate(P):
            a = self.sphere_ab(p[3], p[4], p[5], 1.34, 0.447, cap)
            nmax[j] = a.shape[0] - 1
            ab[j, :a.shape[0], :, 0] = a.real
            ab[j, :a.shape[0], :, 1] = a.imag
        holo = np.zeros(npts, np.float32)
        terms = np.zeros((2, npts), np.float32)
        fp = ctypes.POINTER(ctypes.c_float)
        self.lib.h_hologram_pair(ptr(c), npts, ptr(P), P.shape[0], ptr(ab),
                                 ptr(nmax, _ip), cap, k, 3 | (0 if flag else 8),
                                 ptr(holo, fp), ptr(terms, fp))
        return holo, terms

    def jacobian_aberrated(self, coords, p, ab, dab, k, aberration,
                           bohren=True, fp64=False):
        '''Hologram and Jacobian of the aberrated model of the device fits
        (spherical-aberration coefficient c = aberration).'''
        c = np.ascontiguousarray(coords, dtype=float)
        npts = c.shape[1]
        n, a, d = self._pack_ab(ab, dab)
        holo = np.zeros(npts)
        jac = np.zeros((6, npts))
        pv = np.asarray(p, dtype=float)
        self.lib.h_jacobian_aberrated(ptr(c), npts, ptr(pv), ptr(a), ptr(d), n,
                                      k, 1 | (2 if bohren else 0), int(fp64),
                                      float(aberration), ptr(holo), ptr(jac))
        return holo, jac

    def jacobian_rev(self, coords, p, ab, dab, k, bohren=True, fp64=False):
        '''As jacobian, with the reverse-mode epilogue.'''
        c = np.ascontiguousarray(coords, dtype=float)
        npts = c.shape[1]
        n, a, d = self._pack_ab(ab, dab)
        holo = np.zeros(npts)
        jac = np.zeros((6, npts))
        pv = np.asarray(p, dtype=float)
        self.lib.h_jacobian_rev(ptr(c), npts, ptr(pv), ptr(a), ptr(d), n, k,
                                1 | (2 if bohren else 0), int(fp64),
                                ptr(holo), ptr(jac))
        return holo, jac
