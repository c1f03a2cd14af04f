'''GPU: the differentiable hologram (autograd Function whose backward is the
VJP kernel) and the full 6-column Jacobian, for large spheres too.

References: the pure-torch FP64 autograd restatement of the reference model
(oracle/torch_model.py) and central finite differences of the FP64 oracle.
Tolerances: the chi^2 gradient agrees with the FP64 autograd gradient to
3e-5 of sum_p |g_p| * max_p |dH_p/dparam| (the FP32 Jacobian's relative
accuracy, about 5e-6 of its column maximum, times the sum's size); the
Jacobian agrees with central differences (relative step 1e-5) to 3e-4 of
its column maximum, the reference Jacobian test's tolerance
(tests/test_jaxlorenzmie.py:79-101).
'''
import numpy as np
import pytest
import torch

from oracle import field as ofield, torch_model

pytestmark = pytest.mark.gpu

KEYS = ('x_p', 'y_p', 'z_p', 'a_p', 'n_p', 'k_p')
CASES = [((48, 48), [20.3, 25.7, 120., 0.9, 1.6, 0.01]),
         ((64, 64), [31.5, 30.2, 150., 0.75, 1.45, 0.0]),
         ((64, 64), [31.5, 30.25, 260., 3.0, 1.7, 0.001]),
         ((40, 40), [20.3, 19.6, -130., 0.6, 1.5, 0.0])]


@pytest.mark.parametrize('shape,p', CASES)
def test_chi2_gradient_vs_torch_fp64_autograd(shape, p):
    from pylorenzmie_b200.theory import autograd as ag
    c = ofield.meshgrid(shape)
    ref = ofield.hologram(c, [dict(zip(KEYS, p))], ofield.DEFAULT_INSTRUMENT)
    d = ref + 0.05 * np.random.default_rng(0).normal(size=ref.shape)
    # reference gradient: torch FP64 autograd of the restated model
    pt = torch.tensor(p, dtype=torch.float64, requires_grad=True)
    chi = ((torch_model.hologram(pt, c) - torch.tensor(d)) ** 2).sum()
    chi.backward()
    gref = pt.grad.numpy()
    # ours: forward FP32 kernel, backward VJP kernel
    pg = torch.tensor([p], dtype=torch.float64, device='cuda',
                      requires_grad=True)
    h = ag.hologram(pg, c)
    assert h.shape == (1, c.shape[1]) and h.dtype == torch.float32
    dg = torch.tensor(d, dtype=torch.float32, device='cuda')
    chi_g = ((h[0] - dg) ** 2).sum()
    chi_g.backward()
    g = pg.grad[0].cpu().numpy()
    # bound of the FP32 pixel sum: the Jacobian's relative accuracy times
    # sum_p |2 (H - d)| * max_p |dH/dp|
    _, J = ag.jacobian(pg.detach(), c)
    scale = 2 * np.abs(ref - d).sum() * np.abs(J[0].cpu().numpy()).max(axis=1)
    err = np.abs(g - gref)
    assert np.all(err <= 3e-5 * scale + 1e-9), (err, scale)


def test_vjp_equals_jacobian_transpose_at_large_sizes():
    '''A size-independent identity at the differentiation workload's scale:
    the VJP kernel's sum_p g_p dH_p/dparam equals J^T g from the Jacobian
    kernel (same FP32 pixel math), for 401x401 crops of 3-6 um spheres.'''
    from pylorenzmie_b200 import workloads
    from pylorenzmie_b200.theory import autograd as ag
    P = workloads.large(4, seed=3)
    c = ofield.meshgrid((401, 401))
    pg = torch.tensor(P, dtype=torch.float64, device='cuda',
                      requires_grad=True)
    h = ag.hologram(pg, c)
    gen = torch.Generator(device='cuda').manual_seed(0)
    g = torch.randn(h.shape, generator=gen, device='cuda')
    (h * g).sum().backward()
    vjp = pg.grad.cpu().numpy()
    H, J = ag.jacobian(pg.detach(), c)
    assert torch.isfinite(J).all() and torch.isfinite(H).all()
    jtg = torch.einsum('bjp,bp->bj', J, g.double()).cpu().numpy()
    scale = torch.einsum('bjp,bp->bj', J.abs(), g.double().abs()).cpu().numpy()
    assert np.all(np.abs(vjp - jtg) <= 1e-5 * scale)
    # forward values equal the hologram kernel's: both FP32 sums (the
    # hologram kernel's packed two-pixel loop, the Jacobian kernel's scalar
    # loop), each within 7.7e-6 max(1, H) of the FP64 kernel on these
    # spheres (measured), so within twice that of each other
    hf = h.detach().double().cpu().numpy()
    Hj = H.cpu().numpy()
    assert np.all(np.abs(hf - Hj) <= 2e-5 + 1.5e-5 * np.abs(Hj))


@pytest.mark.parametrize('p', [[50.3, 49.6, 300., 4.0, 1.7, 0.0],
                               [50., 50.5, 420., 5.5, 1.9, 0.0]])
def test_large_sphere_jacobian_vs_finite_differences(p):
    '''Large spheres (n_max 100-200) at a reduced crop: Jacobian columns
    against central differences of the FP64 oracle.  High-index large
    spheres have very sharp resonances (an a_n with |da_n/da_p| ~ 200 /um
    at n = 120 for a_p = 5.5 um, n_p = 1.9), so the radius and index
    steps are 1e-7 relative: at 1e-5 the difference quotient itself is off
    by 100 %.'''
    from pylorenzmie_b200.theory import autograd as ag
    shape = (101, 101)
    c = ofield.meshgrid(shape)
    inst = ofield.DEFAULT_INSTRUMENT
    _, J = ag.jacobian(torch.tensor(p, dtype=torch.float64, device='cuda'),
                       c)
    J = J[0].cpu().numpy()
    for j in range(6):
        step = (1e-5 * abs(p[j]) if j < 3 else
                1e-7 * abs(p[j]) if j < 5 else 1e-8)
        pp, pm = list(p), list(p)
        pp[j] += step
        pm[j] -= step
        fd = (ofield.hologram(c, [dict(zip(KEYS, pp))], inst) -
              ofield.hologram(c, [dict(zip(KEYS, pm))], inst)) / (2 * step)
        err = np.abs(J[j] - fd).max() / np.abs(fd).max()
        assert err < 3e-4, (KEYS[j], err)


def config4_spheres(n, side, seed):
    '''Spheres of the differentiation workload's distribution: a_p
    U(3, 6) um, n_p U(1.4, 2.0), z_p U(200, 600) px (at least 10 px above
    the sphere's top), centred +-2 px on a side x side crop.'''
    rng = np.random.default_rng(seed)
    c = (side - 1) / 2.
    out = []
    for _ in range(n):
        a = rng.uniform(3., 6.)
        out.append([c + rng.uniform(-2, 2), c + rng.uniform(-2, 2),
                    max(rng.uniform(200., 600.), a / 0.048 + 10.), a,
                    rng.uniform(1.4, 2.0), 0.])
    return out


@pytest.mark.parametrize('shape,p', [((201, 201), q) for q in
                                     config4_spheres(3, 201, 41)] +
                         [((401, 401), config4_spheres(1, 401, 42)[0])])
def test_chi2_gradient_vs_torch_fp64_autograd_large(shape, p):
    '''The chi^2 gradient at the differentiation workload's sizes (n_max
    90-190): as test_chi2_gradient_vs_torch_fp64_autograd.'''
    test_chi2_gradient_vs_torch_fp64_autograd(shape, p)


def test_jacobian_vs_torch_fp64_forward_mode_large():
    '''All six Jacobian columns of a 401x401 crop of a large sphere against
    forward-mode derivatives (torch.func.jvp) of the FP64 torch
    restatement, within 5e-5 of each column's maximum.'''
    from pylorenzmie_b200.theory import autograd as ag
    p = config4_spheres(1, 401, 43)[0]
    c = ofield.meshgrid((401, 401))
    _, J = ag.jacobian(torch.tensor(p, dtype=torch.float64, device='cuda'),
                       c)
    J = J[0].cpu().numpy()
    p0 = torch.tensor(p, dtype=torch.float64)
    errs = []
    for j in range(6):
        e = torch.zeros(6, dtype=torch.float64)
        e[j] = 1.
        _, col = torch.func.jvp(lambda q: torch_model.hologram(q, c), (p0,),
                                (e,))
        col = col.numpy()
        errs.append(np.abs(J[j] - col).max() / np.abs(col).max())
    assert max(errs) < 5e-5, dict(zip(KEYS, errs))
