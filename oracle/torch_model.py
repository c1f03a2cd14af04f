'''Pure-torch FP64 autograd restatement of the reference model (oracle).

The reference's torch backend is not differentiable (a_n, b_n come from
numpy and r_p is a fresh non-grad tensor, theory/torchLorenzMie.py:293-300),
and its only Jacobian is JAX ``jacfwd`` (theory/jaxLorenzMie.py:283-286),
which cannot run here.  This module is the substitute gradient reference:
Sphere.mie_coefficients (theory/Sphere.py:147-226) and LorenzMie.lorenzmie
(theory/LorenzMie.py:183-342) written with torch complex128 operations so
that torch.autograd differentiates them, following the structure of the
JAX restatement (theory/jaxLorenzMie.py:26-275: a_n, b_n from (a_p, n_p,
k_p) with n_max fixed, then the per-pixel sum, phase and |E + x|^2).

Test infrastructure only: see ``oracle/__init__.py``.
'''
import math

import torch

from .mie import wiscombe_yang


def mie_ab(a_p, n_p, k_p, n_m, wavelength, nmax):
    '''(nmax+1, 2) complex128 a_n, b_n, differentiable in a_p, n_p, k_p.'''
    k = 2. * math.pi / wavelength * n_m
    x = k * a_p
    m = torch.complex(n_p, k_p) / n_m
    z = x * m
    d1 = [None] * (nmax + 1)
    d = torch.zeros((), dtype=torch.complex128)
    d1[nmax] = d
    for n in range(nmax, 0, -1):
        d = n / z - 1. / (d + n / z)
        d1[n - 1] = d
    xz = x.to(torch.complex128)
    dm = [None] * (nmax + 1)
    d = torch.zeros((), dtype=torch.complex128)
    dm[nmax] = d
    for n in range(nmax, 0, -1):
        d = n / xz - 1. / (d + n / xz)
        dm[n - 1] = d
    psi = [torch.sin(xz)]
    zeta = [-1j * torch.exp(1j * xz)]
    pz = 0.5 * (1. - torch.exp(2j * xz))
    d3 = 1j * torch.ones((), dtype=torch.complex128)
    for n in range(1, nmax + 1):
        t1 = n / xz - dm[n - 1]
        t3 = n / xz - d3
        psi.append(psi[-1] * t1)
        zeta.append(zeta[-1] * t3)
        pz = pz * (t1 * t3)
        d3 = dm[n] + 1j / pz
    rows = [torch.zeros(2, dtype=torch.complex128)]
    for n in range(1, nmax + 1):
        fa = d1[n] / m + n / xz
        a = (fa * psi[n] - psi[n - 1]) / (fa * zeta[n] - zeta[n - 1])
        fb = d1[n] * m + n / xz
        b = (fb * psi[n] - psi[n - 1]) / (fb * zeta[n] - zeta[n - 1])
        rows.append(torch.stack([a, b]))
    return torch.stack(rows)


def hologram(params, coordinates, n_m=1.340, wavelength=0.447,
             magnification=0.048):
    '''Hologram of one sphere, params = (x_p, y_p, z_p, a_p, n_p, k_p)
    float64 tensor (requires_grad allowed); coordinates (2|3, npts).'''
    c = torch.as_tensor(coordinates, dtype=torch.float64)
    if c.shape[0] == 2:
        c = torch.cat([c, torch.zeros(1, c.shape[1], dtype=torch.float64)])
    x_p, y_p, z_p, a_p, n_p, k_p = params.unbind()
    k = 2. * math.pi / wavelength * n_m * magnification
    kkm = 2. * math.pi / wavelength * n_m
    nmax = wiscombe_yang(kkm * float(a_p.detach()),
                         complex(float(n_p.detach()), float(k_p.detach())) / n_m)
    ab = mie_ab(a_p, n_p, k_p, n_m, wavelength, nmax)
    kx = k * (c[0] - x_p)
    ky = k * (c[1] - y_p)
    kz = -k * (c[2] - z_p)
    krho = torch.sqrt(kx * kx + ky * ky)
    kr = torch.sqrt(krho * krho + kz * kz)
    safe = krho > 0
    krs = torch.where(safe, krho, torch.ones_like(krho))
    cosphi = torch.where(safe, kx / krs, torch.ones_like(kx))
    sinphi = torch.where(safe, ky / krs, torch.zeros_like(ky))
    costheta = kz / kr
    sintheta = krho / kr
    sg = 1j * torch.sign(kz)
    xi2 = torch.cos(kr) + sg * torch.sin(kr)
    xi1 = torch.sin(kr) - sg * torch.cos(kr)
    pim1 = torch.zeros_like(kr)
    pi = torch.ones_like(kr)
    es = [torch.zeros_like(xi1) for _ in range(3)]
    fac = 1. + 0j
    for n in range(1, nmax + 1):
        swisc = pi * costheta
        twisc = swisc - pim1
        tau = pim1 - n * twisc
        xi = (2. * n - 1.) * (xi1 / kr) - xi2
        dn = n * (xi / kr) - xi1
        fac = fac * 1j
        en = fac * (2. * n + 1.) / (n * n + n)
        an = 1j * en * ab[n, 0]
        bn = en * ab[n, 1]
        es[0] = es[0] + an * (n * n + n) * pi * xi
        es[1] = es[1] + an * tau * dn - bn * pi * xi
        es[2] = es[2] + an * pi * dn - bn * tau * xi
        pim1, pi = pi, swisc + (1. + 1. / n) * twisc
        xi2, xi1 = xi1, xi
    e0 = es[0] * cosphi * sintheta / kr / kr
    e1 = es[1] * cosphi / kr
    e2 = es[2] * sinphi / kr
    ex = e0 * sintheta * cosphi + e1 * costheta * cosphi - e2 * sinphi
    ey = e0 * sintheta * sinphi + e1 * costheta * sinphi + e2 * cosphi
    ez = e0 * costheta - e1 * sintheta
    phase = torch.exp(-1j * k * z_p)
    ex = ex * phase + 1.
    ey = ey * phase
    ez = ez * phase
    return (ex.abs() ** 2 + ey.abs() ** 2 + ez.abs() ** 2)
