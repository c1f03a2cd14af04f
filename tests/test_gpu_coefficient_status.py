'''GPU: the two-warp coefficient kernels (k_sphere_ab, k_layered_ab) on
launches that mix valid spheres with invalid ones.  Each invalid sphere
gets LMB_ERR_NMAX and zero coefficients; the valid ones get exactly the
coefficients of a launch without the invalid ones (every block is
independent, and both warps of a block pass its barrier on every path).'''
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N_M, LAM = 1.340, 0.447


def _run(fn, *args, n, cap):
    import torch
    from pylorenzmie_b200 import _native
    from pylorenzmie_b200._device import ptr, stream_handle
    lib = _native.load()
    dev = args[0].device
    ab = torch.full((n, cap + 1, 2, 2), 7., dtype=torch.float64, device=dev)
    dab = torch.full((n, cap + 1, 4, 2), 7., dtype=torch.float64, device=dev)
    nmax = torch.full((n,), -5, dtype=torch.int32, device=dev)
    status = torch.full((n,), -5, dtype=torch.int32, device=dev)
    _native.check(getattr(lib, fn)(*[ptr(a) for a in args[:-1]], *args[-1],
                                   N_M, LAM, cap, ptr(ab), ptr(dab), ptr(nmax),
                                   ptr(status), stream_handle(dev)), fn)
    torch.cuda.synchronize()
    return (ab.cpu().numpy(), dab.cpu().numpy(), nmax.cpu().numpy(),
            status.cpu().numpy())


def test_sphere_ab_mixed_valid_and_invalid():
    import torch
    from pylorenzmie_b200 import _native
    rows = [[0., 0., 100., 0.75, 1.42, 0.],      # valid, 26 orders
            [0., 0., 100., -1.0, 1.42, 0.],      # negative radius
            [0., 0., 100., 1.2, math.nan, 0.],   # NaN index
            [0., 0., 100., 3.0, 1.6, 0.],        # n_max above the capacity
            [0., 0., 100., 1.1, 1.55, 0.001]]    # valid, absorbing
    cap = 40
    dev = torch.device('cuda', 0)
    sp = torch.tensor(rows, dtype=torch.float64, device=dev)
    ab, dab, nmax, status = _run('lmb_sphere_ab', sp, (len(rows),),
                                 n=len(rows), cap=cap)
    assert list(status) == [_native.LMB_OK, _native.LMB_ERR_NMAX,
                            _native.LMB_ERR_NMAX, _native.LMB_ERR_NMAX,
                            _native.LMB_OK]
    for i in (1, 2, 3):
        assert not ab[i].any() and not dab[i].any()
    good = torch.tensor([rows[0], rows[4]], dtype=torch.float64, device=dev)
    ab2, dab2, nmax2, status2 = _run('lmb_sphere_ab', good, (2,), n=2,
                                     cap=cap)
    assert list(status2) == [_native.LMB_OK] * 2
    for i, j in ((0, 0), (4, 1)):
        np.testing.assert_array_equal(ab[i], ab2[j])
        np.testing.assert_array_equal(dab[i], dab2[j])
        assert nmax[i] == nmax2[j] > 0


def test_layered_ab_mixed_valid_and_invalid():
    import torch
    from pylorenzmie_b200 import _native
    radii = [[0.3, 0.6, 0.9],       # valid
             [0.6, 0.3, 0.9],       # radii not increasing
             [0.4, 0.8, 1.1],       # valid
             [0.3, 0.6, 4.0]]       # n_max above the capacity
    idx = [[[1.6, 0.], [1.45, 0.002], [1.5, 0.]],
           [[1.6, 0.], [1.45, 0.], [1.5, 0.]],
           [[1.8, 0.01], [1.33, 0.], [1.5, 0.]],
           [[1.6, 0.], [1.45, 0.], [1.5, 0.]]]
    cap = 40
    dev = torch.device('cuda', 0)
    r = torch.tensor(radii, dtype=torch.float64, device=dev)
    ix = torch.tensor(idx, dtype=torch.float64, device=dev)
    ab, dab, nmax, status = _run('lmb_layered_ab', r, ix, (3, len(radii)),
                                 n=len(radii), cap=cap)
    assert list(status) == [_native.LMB_OK, _native.LMB_ERR_NMAX,
                            _native.LMB_OK, _native.LMB_ERR_NMAX]
    for i in (1, 3):
        assert not ab[i].any() and not dab[i].any()
    r2 = torch.tensor([radii[0], radii[2]], dtype=torch.float64, device=dev)
    ix2 = torch.tensor([idx[0], idx[2]], dtype=torch.float64, device=dev)
    ab2, dab2, nmax2, status2 = _run('lmb_layered_ab', r2, ix2, (3, 2), n=2,
                                     cap=cap)
    assert list(status2) == [_native.LMB_OK] * 2
    for i, j in ((0, 0), (2, 1)):
        np.testing.assert_array_equal(ab[i], ab2[j])
        np.testing.assert_array_equal(dab[i], dab2[j])
        assert nmax[i] == nmax2[j] > 0
