'''FP64 restatement of the reference's Lorenz-Mie field and hologram (oracle).

Test infrastructure only: see ``oracle/__init__.py``.
'''
import numpy as np
from .mie import mie_coefficients, layered_coefficients


def meshgrid(shape, corner=(0., 0.), flatten=True):
    '''Pixel grid, lib/meshgrid.py:10-40: (2, ny*nx) as (x, y) rows.'''
    ny, nx = shape
    left, top = corner
    x = np.arange(left, left + nx, dtype=float)
    y = np.arange(top, top + ny, dtype=float)
    xy = np.array(np.meshgrid(x, y))
    return xy.reshape((2, -1)) if flatten else xy


def coordinates3(coordinates):
    '''(ndim, npts) -> (3, npts) with zero z, theory/LorenzMie.py:93-104.'''
    c = np.atleast_2d(np.asarray(coordinates, dtype=float))
    ndim, npts = c.shape
    if ndim > 3:
        raise ValueError(f'Incompatible shape: {c.shape}')
    return np.vstack([c, np.zeros((3 - ndim, npts))])


def wavenumber(n_m, wavelength, magnification):
    '''k in rad/pixel, theory/Instrument.py:46-70 (same operation order).'''
    k = 2. * np.pi / wavelength
    k *= n_m
    k *= magnification
    return k


def lorenzmie(ab, kdr, cartesian=True, bohren=True):
    '''Per-pixel partial-wave sum, theory/LorenzMie.py:183-342.

    Geometry from kdr (kz flipped, :221-237), Riccati-Bessel starting
    values with the sign(kz) convention (:249-251), the n = 1..norders-1
    loop of Wiscombe pi/tau, xi_n, Deirmendjian D_n and the vector
    spherical harmonics (:272-317), geometric factors restored (:322-325)
    and the optional Cartesian projection (:331-340).
    '''
    norders = ab.shape[0]
    kx = kdr[0, :]
    ky = kdr[1, :]
    kz = -kdr[2, :]
    krho = np.hypot(kx, ky)
    kr = np.hypot(krho, kz)
    sinkr = np.sin(kr)
    coskr = np.cos(kr)
    phi = np.arctan2(ky, kx)
    cosphi = np.cos(phi)
    sinphi = np.sin(phi)
    theta = np.arctan2(krho, kz)
    costheta = np.cos(theta)
    sintheta = np.sin(theta)

    factor = 1.j * np.sign(kz) if bohren else -1.j * np.sign(kz)
    xi_nm2 = coskr + factor * sinkr
    xi_nm1 = sinkr - factor * coskr
    pi_nm1 = np.zeros(kx.shape)
    pi_n = np.ones(kx.shape)
    es = np.zeros((3,) + kx.shape, complex)
    prefactor = 1.
    for n in range(1, norders):
        swisc = pi_n * costheta
        twisc = swisc - pi_nm1
        tau_n = pi_nm1 - n * twisc
        xi_n = (2. * n - 1.) * (xi_nm1 / kr) - xi_nm2
        dn = n * (xi_n / kr) - xi_nm1
        mo1 = pi_n * xi_n
        mo2 = tau_n * xi_n
        ne0 = (n * n + n) * mo1
        ne1 = tau_n * dn
        ne2 = pi_n * dn
        prefactor *= 1.j
        en = prefactor * (2. * n + 1.) / (n * n + n)
        an = 1.j * en * ab[n, 0]
        bn = en * ab[n, 1]
        es[0] += an * ne0
        es[1] += an * ne1 - bn * mo1
        es[2] += an * ne2 - bn * mo2
        pi_nm1 = pi_n
        pi_n = swisc + (1. + 1. / n) * twisc
        xi_nm2 = xi_nm1
        xi_nm1 = xi_n

    es[0] *= cosphi * sintheta / kr
    es[1] *= cosphi
    es[2] *= sinphi
    es /= kr
    if not cartesian:
        return es
    ec = np.empty_like(es)
    ec[0] = es[0] * sintheta * cosphi
    ec[0] += es[1] * costheta * cosphi
    ec[0] -= es[2] * sinphi
    ec[1] = es[0] * sintheta * sinphi
    ec[1] += es[1] * costheta * sinphi
    ec[1] += es[2] * cosphi
    ec[2] = es[0] * costheta - es[1] * sintheta
    return ec


def sphere_ab(particle, n_m, wavelength):
    '''ab of a sphere record (dict with a_p, n_p, k_p) or a layered record
    (dict with 'layers': (radii, indices)).'''
    if 'layers' in particle:
        radii, indices = particle['layers']
        return layered_coefficients(radii, indices, n_m, wavelength)
    return mie_coefficients(particle['a_p'], particle['n_p'],
                            particle.get('k_p', 0.), n_m, wavelength)


def scattered_field(coordinates, particle, instrument, cartesian=True,
                    bohren=True):
    '''One particle's field incl. exp(-i k z_p), theory/LorenzMie.py:135-158.

    ``particle`` is a dict with x_p, y_p, z_p and either a_p/n_p/k_p or
    'layers'; ``instrument`` is a dict with n_m, wavelength, magnification.
    '''
    k = wavenumber(instrument['n_m'], instrument['wavelength'],
                   instrument['magnification'])
    r_p = np.array([particle['x_p'], particle['y_p'], particle['z_p']])
    kdr = k * (coordinates - r_p[:, None])
    ab = sphere_ab(particle, instrument['n_m'], instrument['wavelength'])
    return lorenzmie(ab, kdr, cartesian, bohren) * np.exp(-1.j * k * r_p[2])


def field(coordinates, particles, instrument, cartesian=True, bohren=True):
    '''Superposed field of a particle list, theory/LorenzMie.py:160-181.'''
    c = coordinates3(coordinates)
    out = np.zeros(c.shape, complex)
    for p in particles:
        out += scattered_field(c, p, instrument, cartesian, bohren)
    return out


def hologram(coordinates, particles, instrument, cartesian=True, bohren=True):
    '''Hologram sum_c |E_c + delta_cx|^2, theory/LorenzMie.py:113-133.'''
    f = field(coordinates, particles, instrument, cartesian, bohren)
    f[0, :] += 1.
    return np.sum(f.real ** 2 + f.imag ** 2, axis=0)


DEFAULT_INSTRUMENT = dict(wavelength=0.447, magnification=0.048,
                          n_m=1.340, numerical_aperture=1.45, noise=0.05)


def aberrated_hologram(coordinates, particles, instrument, spherical,
                       cartesian=True, bohren=True):
    '''Hologram of AberratedLorenzMie (theory/Aberrated.py:62-85): each
    particle's scattered field times exp(i Phi), Phi = (4 n_m^3 / k) s
    r^4 / (r^2 + z_p^2)^2 with r the in-plane distance from the particle
    (pixels) and z_p its axial position.'''
    c = coordinates3(coordinates)
    k = wavenumber(instrument['n_m'], instrument['wavelength'],
                   instrument['magnification'])
    out = np.zeros(c.shape, complex)
    for p in particles:
        f = scattered_field(c, p, instrument, cartesian, bohren)
        if spherical != 0.:
            x = c[0] - p['x_p']
            y = c[1] - p['y_p']
            rsq = x * x + y * y
            phase = (4. * instrument['n_m'] ** 3 / k) * spherical * \
                rsq ** 2 / (rsq + p['z_p'] ** 2) ** 2
            f = f * np.exp(1j * phase)
        out += f
    out[0, :] += 1.
    return np.sum(out.real ** 2 + out.imag ** 2, axis=0)
