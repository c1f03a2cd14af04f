'''lmb_fit_batch_noalloc: the batched fit for callers that cannot allocate
device memory (a real-time acquisition loop, or a host that owns all device
memory through another allocator), checked through the C ABI against the
regular lmb_fit_batch on the same inputs, on two calls in a row.

This file is collected last on purpose (test_zz_*), so a run that stops at
its first failure has run every other test before it.
'''
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# same tolerances as the fit parity tests (tests/test_gpu_fit.py)
TOL = np.array([0.02, 0.02, 0.02, 1e-3, 1e-4, 1e-4])


def _noalloc(lib):
    fn = lib.lmb_fit_batch_noalloc
    vp, d = ctypes.c_void_p, ctypes.c_double
    fn.restype = ctypes.c_int
    fn.argtypes = [vp, ctypes.c_int, ctypes.c_longlong, vp, vp, vp, d, d, d,
                   d, ctypes.c_int, ctypes.c_void_p, vp, vp]
    return fn


def _batch(seed, shape=(61, 61), B=6):
    from pylorenzmie_b200 import workloads
    rng = np.random.default_rng(seed)
    c = (shape[0] - 1) / 2.
    truth = np.zeros((B, 6))
    truth[:, 0] = c + rng.uniform(-2, 2, B)
    truth[:, 1] = c + rng.uniform(-2, 2, B)
    truth[:, 2] = rng.uniform(150., 250., B)
    truth[:, 3] = rng.uniform(0.5, 1.0, B)
    truth[:, 4] = rng.uniform(1.38, 1.6, B)
    start = truth.copy()
    start[:, 2] += 10.
    start[:, 3] *= 1.05
    start[:, 4] += 0.02
    data = workloads.render(truth, shape, seed=seed).cpu().numpy()
    return data, start


def _run_both(data, start):
    import torch
    from pylorenzmie_b200 import _native, Instrument
    from pylorenzmie_b200.analysis import _fit
    lib = _native.load()
    inst = Instrument()
    B, ny, nx = data.shape
    packed = _fit.PackedFeatures([(data[i], (0., 0., ny, nx), None)
                                  for i in range(B)])
    variables = ['x_p', 'y_p', 'z_p', 'a_p', 'n_p']
    cap = _fit.fit_capacity(start, inst.n_m, inst.wavelength)

    # regular entry point, caller-provided workspace
    d_feat, d_data, _, d_params = _fit.upload(packed, start)
    d_res, _ = _fit.fit_device(d_feat, d_data, None, d_params, B,
                               packed.total, inst, variables, None, cap,
                               start)
    p_ref = d_params.view(torch.float64).reshape(B, 6).cpu().numpy()
    r_ref = d_res[:B * 80].cpu().numpy().view(_native.RESULT_DTYPE).copy()

    # no-allocation entry point, same device inputs, fresh start values
    d_params2 = torch.from_numpy(np.ascontiguousarray(start)).to(d_data.device)
    d_res2 = torch.zeros(B * 80, dtype=torch.uint8, device=d_data.device)
    st = _native.FitSettings()
    st.ftol, st.xtol, st.gtol, st.factor = 1e-4, 1e-6, 1e-6, 100.
    st.max_nfev = 2000
    st.variables = _fit.variable_mask(variables)
    st.flags = _native.LMB_BOHREN
    st.max_iterations = 2000
    status = _noalloc(lib)(
        d_feat.data_ptr(), B, packed.total, d_data.data_ptr(), None,
        d_params2.data_ptr(), inst.n_m, inst.wavelength, inst.magnification,
        inst.noise, cap, ctypes.addressof(st), d_res2.data_ptr(),
        torch.cuda.current_stream().cuda_stream)
    assert status == _native.LMB_OK, _native.status_string(status)
    p_new = d_params2.cpu().numpy()
    r_new = d_res2.cpu().numpy().view(_native.RESULT_DTYPE).copy()
    return p_ref, r_ref, p_new, r_new


def test_noalloc_matches_regular_fit_twice():
    # two calls in a row with different inputs: the shared static scratch
    # keeps the first call's contents, which must not leak into the second
    for seed in (11, 12):
        data, start = _batch(seed)
        p_ref, r_ref, p_new, r_new = _run_both(data, start)
        assert np.all(r_ref['success'] == 1) and np.all(r_new['success'] == 1)
        assert np.all(np.abs(p_new - p_ref) <= TOL), (p_new - p_ref)
        np.testing.assert_array_equal(r_new['status'], r_ref['status'])
        np.testing.assert_array_equal(r_new['nfev'], r_ref['nfev'])
        np.testing.assert_allclose(r_new['redchi'], r_ref['redchi'],
                                   rtol=1e-6)
        np.testing.assert_allclose(r_new['dparams'], r_ref['dparams'],
                                   rtol=1e-4, atol=1e-12)


def test_noalloc_rejects_requests_above_its_scratch():
    import torch
    from pylorenzmie_b200 import _native
    lib = _native.load()
    st = _native.FitSettings()
    st.ftol, st.xtol, st.gtol, st.factor = 1e-4, 1e-6, 1e-6, 100.
    st.max_nfev = st.max_iterations = 10
    st.variables = 31
    st.flags = _native.LMB_BOHREN
    nf, total = 4000, 4000 * 201 * 201
    need = lib.lmb_fit_workspace_bytes(nf, total, 40)
    assert need > LIMIT
    # valid buffers for every record the call could touch: zero-pixel
    # features, so nothing would read the (small) data buffer even if the
    # size check were missing
    dev = torch.device('cuda')
    feat = np.zeros(nf, dtype=_native.FEATURE_DTYPE)
    d_feat = torch.from_numpy(feat.view(np.uint8).copy()).to(dev)
    d_data = torch.zeros(16, dtype=torch.float32, device=dev)
    d_params = torch.zeros((nf, 6), dtype=torch.float64, device=dev)
    d_res = torch.zeros(nf * 80, dtype=torch.uint8, device=dev)
    status = _noalloc(lib)(d_feat.data_ptr(), nf, total, d_data.data_ptr(),
                           None, d_params.data_ptr(), 1.34, 0.447, 0.048,
                           0.05, 40, ctypes.addressof(st), d_res.data_ptr(),
                           torch.cuda.current_stream().cuda_stream)
    assert status == _native.LMB_ERR_WORKSPACE
    torch.cuda.synchronize()


LIMIT = 16 * 1024 * 1024
