'''The C-ABI library: it loads without a GPU, exports every entry point that
include/lmb200.h declares, and its struct layouts match the host mirror.
No compute runs here (only calls that return before touching CUDA).'''
import ctypes
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from pylorenzmie_b200 import _native, build

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    text = '\n'.join(p.read_text() for p in sorted((ROOT / 'include').glob('*.h')))
    text = re.sub(r'/\*.*?\*/', '', text, flags=re.S)
    return sorted(set(re.findall(r'\b(lmb_\w+)\s*\(', text)))


@pytest.fixture(scope='module')
def lib():
    return _native.load()


def test_library_is_in_tree_and_sm100a(lib):
    path = _native.library_path()
    assert path.exists() and path.parent == ROOT / 'pylorenzmie_b200' / '_lib'
    cmd = build.command()
    assert 'arch=compute_100a,code=sm_100a' in ' '.join(cmd)


def test_exports_every_declared_symbol(lib):
    syms = declared_symbols()
    assert len(syms) >= 12
    out = subprocess.run(['nm', '-D', '--defined-only',
                          str(_native.library_path())],
                         capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r' T (\w+)', out))
    missing = [s for s in syms if s not in exported]
    assert not missing, missing
    for s in syms:
        getattr(lib, s)
    assert set(_native.symbols()) <= set(syms)


def test_version_and_status_strings(lib):
    assert lib.lmb_version() == 100
    for st in range(6):
        assert isinstance(_native.status_string(st), str)
    assert 'workspace' in _native.status_string(_native.LMB_ERR_WORKSPACE)


def test_struct_layouts():
    assert _native.SPHERE_DTYPE.itemsize == 48
    assert _native.FEATURE_DTYPE.itemsize == 40
    assert _native.RESULT_DTYPE.itemsize == 80
    assert ctypes.sizeof(_native.FitSettings) == 56
    assert ctypes.sizeof(_native.FitStats) == 48


def test_argument_checks_without_gpu(lib):
    # these return before any CUDA call
    assert lib.lmb_sphere_ab(None, 0, 1.34, 0.447, 10, None, None, None,
                             None, None) == _native.LMB_OK
    assert lib.lmb_sphere_ab(None, 1, 1.34, 0.447, 0, None, None, None,
                             None, None) == _native.LMB_ERR_ARG
    assert lib.lmb_sphere_ab(None, 1, 1.34, 0.447, 10, None, None, None,
                             None, None) == _native.LMB_ERR_ARG
    assert lib.lmb_hologram(None, 0, None, None, 0, None, None, 10, 1., 3,
                            None, None) == _native.LMB_OK
    assert lib.lmb_hologram(None, 10, None, None, 1, None, None, 10, 1., 3,
                            None, None) == _native.LMB_ERR_ARG
    assert lib.lmb_jacobian(None, 0, None, 0, None, None, None, 10, 1., 3,
                            None, None, None) == _native.LMB_OK
    st = _native.FitSettings()
    assert lib.lmb_fit_batch(None, 0, 0, None, None, None, 1.34, 0.447,
                             0.048, 0.05, 10, st, None, None, 0, None,
                             None) == _native.LMB_OK
    assert lib.lmb_fit_batch(None, 2, 10, None, None, None, 1.34, 0.447,
                             0.048, 0.05, 10, st, None, None, 0, None,
                             None) == _native.LMB_ERR_ARG


def test_argument_checks_of_the_search_and_variant_entry_points(lib):
    '''The device differential evolution, the crops chi^2 and the
    aberrated entry points reject bad sizes and coefficients before any
    device work (no GPU needed for these answers).'''
    nan = float('nan')
    ARG, OK = _native.LMB_ERR_ARG, _native.LMB_OK
    # lmb_de_trial: nsearch, npop >= 3, nparam 1..6, mutation in [0, 2)
    def trial(ns, nl, npop, npar):
        return lib.lmb_de_trial(ns, nl, None, npop, npar, None, None, None, 0,
                                0.5, 1., None, None, None, None, None, None,
                                0, None, None)

    def select(ns, nl, npop, npar):
        return lib.lmb_de_select(ns, nl, None, npop, npar, None, None, None,
                                 None, None, None, None, None, None, 0, None)
    assert trial(4, 0, 10, 3) == OK and select(4, 0, 10, 3) == OK
    for args in ((-1, 0, 10, 3), (2, 3, 10, 3), (2, 2, 2, 3), (2, 2, 10, 0),
                 (2, 2, 10, 7), (2, 2, 10, 3)):    # the last: null buffers
        assert trial(*args) == ARG and select(*args) == ARG, args
    # lmb_de_shuffles (host): a bit generator is required, keep <= n
    idx = np.arange(4, dtype=np.int64)
    out = np.zeros((2, 3), dtype=np.int64)
    assert lib.lmb_de_shuffles(None, idx.ctypes.data, 4, 2, 3,
                               out.ctypes.data) == ARG
    bg = np.random.default_rng(0).bit_generator
    assert lib.lmb_de_shuffles(bg.ctypes.bit_generator, idx.ctypes.data, 4,
                               2, 5, out.ctypes.data) == ARG
    assert lib.lmb_de_shuffles(bg.ctypes.bit_generator, idx.ctypes.data, 4,
                               0, 3, None) == OK
    # lmb_de_draws (host): n >= 1, keep <= n, nparam >= 1, buffers
    fill = np.zeros(4, dtype=np.int64)
    cross = np.zeros((4, 2), dtype=bool)
    first = np.zeros((4, 3), dtype=np.int64)
    def draws(n, keep, npar, fb=fill.ctypes.data):
        return lib.lmb_de_draws(bg.ctypes.bit_generator, 1, 0, 0., 0., None,
                                idx.ctypes.data, n, keep, first.ctypes.data,
                                npar, 0.7, fb, cross.ctypes.data)
    assert draws(0, 0, 2) == ARG and draws(4, 5, 2) == ARG
    assert draws(4, 3, 0) == ARG and draws(4, 3, 2, None) == ARG
    assert lib.lmb_de_draws(bg.ctypes.bit_generator, 1, 1, 0.5, 1., None,
                            idx.ctypes.data, 4, 3, first.ctypes.data, 2, 0.7,
                            fill.ctypes.data, cross.ctypes.data) == ARG
    assert lib.lmb_de_draws_many(0, None, None, None, None, None, None,
                                 None, 4, 3, None, 2, None, None, None) == OK
    assert lib.lmb_de_draws_many(2, None, None, None, None, None, None,
                                 None, 4, 3, None, 2, None, None, None) == ARG
    # lmb_chi2_crops: no items is a no-op; items without crops are not
    assert lib.lmb_chi2_crops(None, 0, None, 0.05, None, 0, None, 0, None,
                              None, 0, None, None, 10, 1., 3, None, None,
                              None, 0, None, 0.) == OK
    assert lib.lmb_chi2_crops(None, 10, None, 0.05, None, 0, None, 5, None,
                              None, 2, None, None, 10, 1., 3, None, None,
                              None, 0, None, 0.) == ARG
    # non-finite aberration coefficients
    assert lib.lmb_jacobian_aberrated(None, 0, None, 0, None, None, None, 10,
                                      1., 3, nan, None, None, None) == ARG
    assert lib.lmb_jacobian_aberrated(None, 0, None, 0, None, None, None, 10,
                                      1., 3, 2.5, None, None, None) == OK
    st = _native.FitSettings()
    assert lib.lmb_fit_batch_aberrated(None, 0, 0, None, None, None, 1, None,
                                       None, 1.34, 0.447, 0.048, 0.05, 10,
                                       2.5, st, None, None, 0, None,
                                       None) == OK
    assert lib.lmb_fit_batch_aberrated(None, 2, 10, None, None, None, 1,
                                       None, None, 1.34, 0.447, 0.048, 0.05,
                                       10, 2.5, st, None, None, 0, None,
                                       None) == ARG


def test_workspace_sizes(lib):
    a = lib.lmb_fit_workspace_bytes(256, 256 * 201 * 201, 40)
    b = lib.lmb_fit_workspace_bytes(512, 512 * 201 * 201, 40)
    assert 0 < a < b
    assert a % 256 == 0
    assert lib.lmb_fit_workspace_bytes(0, 0, 40) == 0
    assert lib.lmb_vjp_workspace_bytes(1000, 2) == 8 * 2 * 6 * 8
    assert lib.lmb_vjp_workspace_bytes(0, 2) == 0



def test_pack_crops_host_conversion():
    '''lmb_pack_crops (host code, no GPU): many crops of float64 or float32,
    any lengths, on several native threads: numpy's float32 rounding, in
    order, nothing written outside the destination run.'''
    lib = _native.load()
    rng = np.random.default_rng(5)
    for dtype, kind in ((np.float64, _native.LMB_PACK_F64),
                        (np.float32, _native.LMB_PACK_F32)):
        for sizes in ([0, 1, 7], [300000, 5, 0, 700001, 3],
                      list(rng.integers(0, 40000, 200))):
            srcs = [rng.normal(0., 3., n).astype(dtype) for n in sizes]
            ptrs = np.array([s.ctypes.data for s in srcs], dtype=np.uintp)
            counts = np.array(sizes, dtype=np.int64)
            total = int(counts.sum())
            out = np.full(total + 5, -7., np.float32)
            for threads in (1, 6):
                out[:] = -7.
                assert lib.lmb_pack_crops(ptrs.ctypes.data,
                                          counts.ctypes.data, len(srcs), kind,
                                          out[2:].ctypes.data, threads) == 0
                ref = np.concatenate(srcs).astype(np.float32) if srcs else []
                np.testing.assert_array_equal(out[2:2 + total], ref)
                assert np.all(out[:2] == -7.) and np.all(out[2 + total:] == -7.)
    ptrs = np.zeros(1, dtype=np.uintp)
    counts = np.array([4], dtype=np.int64)
    out = np.zeros(4, np.float32)
    assert lib.lmb_pack_crops(ptrs.ctypes.data, counts.ctypes.data, 1,
                              _native.LMB_PACK_F64, out.ctypes.data, 2) == \
        _native.LMB_ERR_ARG          # null source with a positive count
    assert lib.lmb_pack_crops(ptrs.ctypes.data, counts.ctypes.data, 1, 7,
                              out.ctypes.data, 2) == _native.LMB_ERR_ARG
