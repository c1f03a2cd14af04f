'''FP64 restatement of the reference's Mie-coefficient algorithms (oracle).

Test infrastructure only: see ``oracle/__init__.py``.
'''
import numpy as np


def wiscombe_yang(x, m):
    '''Number of partial waves, theory/Sphere.py:91-123.

    Wiscombe (1980) n_s from the outer size parameter, then Yang (2003)
    Eq. (30): the maximum of n_s, |x m| and |roll(x, -1) m|.  For a scalar x
    the roll is x itself (theory/Sphere.py:120-122).
    '''
    x = np.atleast_1d(np.asarray(x, dtype=float))
    m = np.atleast_1d(np.asarray(m, dtype=complex))
    xl = abs(x[-1])
    if xl <= 8.:
        ns = np.floor(xl + 4. * np.cbrt(xl) + 1.)
    elif xl <= 4200.:
        ns = np.floor(xl + 4.05 * np.cbrt(xl) + 2.)
    else:
        ns = np.floor(xl + 4. * np.cbrt(xl) + 2.)
    xm = np.abs(x * m)
    xm_1 = np.abs(np.roll(x, -1) * m)
    return int(max(ns, xm.max(), xm_1.max()))


def neves_pisignano(x, precision=6.):
    '''Alternative truncation, theory/Sphere.py:125-145.'''
    return int(x + 0.76 * np.cbrt(precision * precision * x) - 4.1)


def mie_coefficients(a_p, n_p, k_p, n_m, wavelength):
    '''a_n, b_n of a homogeneous sphere, theory/Sphere.py:147-226.

    Zero-start downward recurrence for the logarithmic derivative D1 inside
    the sphere (z = m x) and in the medium (z = x); upward recurrences for
    psi, zeta, psi*zeta and D3; Eqs. (5)/(6) of Pena & Pal (2009).
    Returns complex128 of shape (nmax+1, 2) with row 0 zero.
    '''
    k = 2. * np.pi / wavelength
    k *= np.real(n_m)
    x = k * a_p
    m = (n_p + 1.j * k_p) / n_m
    nmax = wiscombe_yang(x, m)

    d1_in = np.zeros(nmax + 1, complex)
    z = x * m
    for n in range(nmax, 0, -1):
        d1_in[n - 1] = n / z - 1. / (d1_in[n] + n / z)

    d1 = np.zeros(nmax + 1, complex)
    z = complex(x)
    for n in range(nmax, 0, -1):
        d1[n - 1] = n / z - 1. / (d1[n] + n / z)

    psi = np.zeros(nmax + 1, complex)
    zeta = np.zeros(nmax + 1, complex)
    d3 = np.zeros(nmax + 1, complex)
    psi[0] = np.sin(z)
    zeta[0] = -1.j * np.exp(1.j * z)
    psizeta = 0.5 * (1. - np.exp(2.j * z))
    d3[0] = 1.j
    for n in range(1, nmax + 1):
        psi[n] = psi[n - 1] * (n / z - d1[n - 1])
        zeta[n] = zeta[n - 1] * (n / z - d3[n - 1])
        psizeta *= (n / z - d1[n - 1]) * (n / z - d3[n - 1])
        d3[n] = d1[n] + 1.j / psizeta

    ab = np.empty((nmax + 1, 2), complex)
    n = np.arange(nmax + 1)
    psi_prev = np.roll(psi, 1)
    zeta_prev = np.roll(zeta, 1)
    fac = d1_in / m + n / x
    ab[:, 0] = (fac * psi - psi_prev) / (fac * zeta - zeta_prev)
    fac = d1_in * m + n / x
    ab[:, 1] = (fac * psi - psi_prev) / (fac * zeta - zeta_prev)
    ab[0, :] = 0.j
    return ab


def layered_coefficients(a_p, n_p, n_m, wavelength):
    '''a_n, b_n of a multilayer sphere (Yang 2003), FP64.

    Restates lib/obsolete/sphere_coefficients.py:65-220 with its input
    handling repaired (the reference wraps list input in an extra dimension
    at :85-89 and calls ``max`` on arrays at :61): radii ``a_p`` and
    indices ``n_p`` are 1-D arrays ordered from the core outwards,
    ``nlayers = len(a_p)`` and nstop follows wiscombe_yang above.  The
    resolution cut of :216-218 is not applied (resolution=None).
    '''
    a_p = np.atleast_1d(np.asarray(a_p, dtype=float))
    n_p = np.atleast_1d(np.asarray(n_p, dtype=complex))
    nlayers = a_p.size
    if n_p.size != nlayers:
        raise ValueError('a_p and n_p must have the same number of elements')
    k = 2. * np.pi * np.real(n_m) / wavelength
    x = k * a_p
    m = n_p / n_m
    nmax = wiscombe_yang(x, m)

    d1_a = np.zeros((nmax + 2, nlayers), complex)
    d1_am1 = np.zeros((nmax + 2, nlayers), complex)
    d3_a = np.zeros((nmax + 1, nlayers), complex)
    d3_am1 = np.zeros((nmax + 1, nlayers), complex)
    pz_a = np.zeros((nmax + 1, nlayers), complex)
    pz_am1 = np.zeros((nmax + 1, nlayers), complex)
    q = np.zeros((nmax + 1, nlayers), complex)
    ha = np.zeros((nmax + 1, nlayers), complex)
    hb = np.zeros((nmax + 1, nlayers), complex)

    # core, sphere_coefficients.py:126-142 (D1 starts at nmax+1)
    z1 = x[0] * m[0]
    for n in range(nmax + 1, 0, -1):
        d1_a[n - 1, 0] = n / z1 - 1. / (d1_a[n, 0] + n / z1)
    pz_a[0, 0] = 0.5 * (1. - np.exp(2.j * z1))
    d3_a[0, 0] = 1.j
    for n in range(1, nmax + 1):
        pz_a[n, 0] = pz_a[n - 1, 0] * (n / z1 - d1_a[n - 1, 0]) * \
            (n / z1 - d3_a[n - 1, 0])
        d3_a[n, 0] = d1_a[n, 0] + 1.j / pz_a[n, 0]
    ha[:, 0] = d1_a[:-1, 0]
    hb[:, 0] = d1_a[:-1, 0]

    # shells, sphere_coefficients.py:144-190
    for ii in range(1, nlayers):
        z1 = x[ii] * m[ii]
        z2 = x[ii - 1] * m[ii]
        for n in range(nmax + 1, 0, -1):
            d1_a[n - 1, ii] = n / z1 - 1. / (d1_a[n, ii] + n / z1)
            d1_am1[n - 1, ii] = n / z2 - 1. / (d1_am1[n, ii] + n / z2)
        pz_a[0, ii] = 0.5 * (1. - np.exp(2.j * z1))
        pz_am1[0, ii] = 0.5 * (1. - np.exp(2.j * z2))
        d3_a[0, ii] = 1.j
        d3_am1[0, ii] = 1.j
        for n in range(1, nmax + 1):
            pz_a[n, ii] = pz_a[n - 1, ii] * (n / z1 - d1_a[n - 1, ii]) * \
                (n / z1 - d3_a[n - 1, ii])
            pz_am1[n, ii] = pz_am1[n - 1, ii] * \
                (n / z2 - d1_am1[n - 1, ii]) * (n / z2 - d3_am1[n - 1, ii])
            d3_a[n, ii] = d1_a[n, ii] + 1.j / pz_a[n, ii]
            d3_am1[n, ii] = d1_am1[n, ii] + 1.j / pz_am1[n, ii]
        q[0, ii] = (np.exp(-2.j * z2) - 1.) / (np.exp(-2.j * z1) - 1.)
        for n in range(1, nmax + 1):
            num = (z1 * d1_a[n, ii] + n) * (n - z1 * d3_a[n - 1, ii])
            den = (z2 * d1_am1[n, ii] + n) * (n - z2 * d3_am1[n - 1, ii])
            q[n, ii] = (x[ii - 1] / x[ii]) ** 2 * q[n - 1, ii] * num / den
        for n in range(1, nmax + 1):
            g1 = m[ii] * ha[n, ii - 1] - m[ii - 1] * d1_am1[n, ii]
            g2 = m[ii] * ha[n, ii - 1] - m[ii - 1] * d3_am1[n, ii]
            temp = q[n, ii] * g1
            ha[n, ii] = (g2 * d1_a[n, ii] - temp * d3_a[n, ii]) / (g2 - temp)
            g1 = m[ii - 1] * hb[n, ii - 1] - m[ii] * d1_am1[n, ii]
            g2 = m[ii - 1] * hb[n, ii - 1] - m[ii] * d3_am1[n, ii]
            temp = q[n, ii] * g1
            hb[n, ii] = (g2 * d1_a[n, ii] - temp * d3_a[n, ii]) / (g2 - temp)

    # medium, sphere_coefficients.py:192-215 (D1 starts at nmax)
    z1 = complex(x[-1])
    d1 = np.zeros(nmax + 2, complex)
    for n in range(nmax, 0, -1):
        d1[n - 1] = n / z1 - 1. / (d1[n] + n / z1)
    psi = np.zeros(nmax + 1, complex)
    zeta = np.zeros(nmax + 1, complex)
    d3 = np.zeros(nmax + 1, complex)
    psi[0] = np.sin(z1)
    zeta[0] = -1.j * np.exp(1.j * z1)
    psizeta = 0.5 * (1. - np.exp(2.j * z1))
    d3[0] = 1.j
    for n in range(1, nmax + 1):
        psi[n] = psi[n - 1] * (n / z1 - d1[n - 1])
        zeta[n] = zeta[n - 1] * (n / z1 - d3[n - 1])
        psizeta = psizeta * (n / z1 - d1[n - 1]) * (n / z1 - d3[n - 1])
        d3[n] = d1[n] + 1.j / psizeta

    n = np.arange(nmax + 1)
    ab = np.empty((nmax + 1, 2), complex)
    fac = ha[:, -1] / m[-1] + n / x[-1]
    ab[:, 0] = (fac * psi - np.roll(psi, 1)) / (fac * zeta - np.roll(zeta, 1))
    fac = hb[:, -1] * m[-1] + n / x[-1]
    ab[:, 1] = (fac * psi - np.roll(psi, 1)) / (fac * zeta - np.roll(zeta, 1))
    ab[0, :] = 0.j
    return ab
