'''Drop-in Lorenz-Mie generative model on the B200 kernels.

``LorenzMie`` keeps the reference's constructor and methods
(theory/LorenzMie.py:52-181): ``coordinates``, ``particle``,
``instrument``, ``properties``, ``field()``, ``hologram()``,
``scattered_field()``; the batched ``batch_field``/``batch_hologram`` of
TorchLorenzMieBatch (theory/torchLorenzMieBatch.py:258-373); and the
analytic-Jacobian slot ``jac()``/``jac_params`` of jaxLorenzMie
(theory/jaxLorenzMie.py:321, 354-395), here covering k_p too.

``method = 'b200 numpy'`` contains 'numpy', so the reference's own
Optimizer (analysis/Optimizer.py:54, 64-65) accepts this model as well.

All compute runs in the CUDA library: Mie coefficients in FP64, the
per-pixel sums in FP32 (``double_precision=True`` selects the FP64 sums).
Results come back as numpy float64/complex128 by default, like the
reference; ``device=True`` returns the CUDA tensor instead (the precedent
of cupyLorenzMie, theory/cupyLorenzMie.py:80, 100).
'''
import numpy as np
import torch

from ..lib import LMObject
from .._device import get_device
from .Sphere import Sphere
from .Instrument import Instrument
from . import _kernels as K

JAC_KEYS = ('x_p', 'y_p', 'z_p', 'a_p', 'n_p', 'k_p')


def _row(p):
    # plain attribute reads where the particle has them (r_p and r_0
    # build arrays)
    try:
        r = (p.x_p + p.x_0, p.y_p + p.y_0, p.z_p + p.z_0)
    except AttributeError:
        r = np.asarray(p.r_p, dtype=float) + np.asarray(
            getattr(p, 'r_0', (0., 0., 0.)), dtype=float)
    return (float(r[0]), float(r[1]), float(r[2]), float(p.a_p),
            float(p.n_p), float(getattr(p, 'k_p', 0.)))


def _records(particles):
    '''SPHERE_DTYPE records (r_p + r_0, a_p, n_p, k_p) of a particle list.'''
    return np.array([_row(p) for p in particles], dtype=K.SPHERE_DTYPE)


class LorenzMie(LMObject):
    '''Scattered field and hologram of one or more spheres.

    Parameters
    ----------
    coordinates : array (2|3, npts), optional. Default: 201x201 grid.
    particle : Sphere or list of Sphere, optional. Default: Sphere().
    instrument : Instrument, optional.
    double_precision : bool. FP64 per-pixel sums (default FP32 sums with
        FP64 Mie coefficients).
    device : torch device spec of a CUDA device. Default: current device.
    '''

    method: str = 'b200 numpy'
    jac_params: frozenset = frozenset(JAC_KEYS)

    def __init__(self, coordinates=None, particle=None, instrument=None,
                 double_precision=False, device=None):
        super().__init__()
        self._device_spec = device
        self._device = None
        self.double_precision = bool(double_precision)
        self.coordinates = coordinates
        self.particle = particle or Sphere()
        self.instrument = instrument or Instrument()

    def __repr__(self):
        classname = self.__class__.__qualname__
        r = f'{classname}(instrument, particle)'
        inst = f'instrument={self.instrument!r}'.replace(',', ',\n\t')
        part = f'particle={self.particle!r}'.replace(',', ',\n\t')
        return '\n    '.join([r, inst, part])

    @property
    def device(self):
        '''The CUDA device; resolved on first use (RuntimeError without a
        GPU, as theory/torchLorenzMie.py:178-201).'''
        if self._device is None:
            self._device = get_device(self._device_spec)
        return self._device

    # properties protocol, theory/LorenzMie.py:68-81
    @property
    def properties(self):
        return {**self.particle.properties, **self.instrument.properties}

    @properties.setter
    def properties(self, properties):
        for name, value in properties.items():
            if hasattr(self.particle, name):
                setattr(self.particle, name, value)
            elif hasattr(self.instrument, name):
                setattr(self.instrument, name, value)
            elif hasattr(self, name):
                setattr(self, name, value)

    # coordinates, theory/LorenzMie.py:83-111
    @property
    def coordinates(self):
        return self._coordinates

    @coordinates.setter
    def coordinates(self, coordinates):
        if coordinates is None:
            c = self.meshgrid((201, 201))
        else:
            c = np.atleast_2d(np.asarray(coordinates, dtype=float))
        ndim, npts = c.shape
        if ndim > 3:
            raise ValueError(f'Incompatible shape: {c.shape=}')
        self._coordinates = np.vstack([c, np.zeros((3 - ndim, npts))])
        self._allocate()

    def _allocate(self):
        '''Invalidate the device copy of the coordinates.'''
        self._coords_dev = None

    @property
    def _coords(self):
        '''Device copy of the coordinates, (3, npts) float64.'''
        if self._coords_dev is None:
            self._coords_dev = torch.from_numpy(
                np.ascontiguousarray(self._coordinates)).to(self.device)
        return self._coords_dev

    # ------------------------------------------------------------------
    def _prepare(self, particle_lists, deriv=False):
        '''Device spheres, item offsets and Mie coefficients.'''
        flat = [p for plist in particle_lists for p in plist]
        inst = self.instrument
        counts = [len(pl) for pl in particle_lists]
        item_start = K.to_device_async(
            np.concatenate([[0], np.cumsum(counts)]).astype(np.int32),
            self.device)
        rec = _records(flat)
        if len(flat) == 0:
            cap = 1
        elif not any(K.is_layered(p) for p in flat):
            cap = int(K.wiscombe_yang(rec['a_p'], rec['n_p'], rec['k_p'],
                                      inst.n_m, inst.wavelength).max()) + 2
        else:
            cap = max(K.particle_nmax(p, inst.n_m, inst.wavelength)
                      for p in flat) + 2
        if cap > K._native.LMB_NMAX_LIMIT:
            raise ValueError(f'a particle needs {cap - 2} partial-wave '
                             f'orders; the limit is '
                             f'{K._native.LMB_NMAX_LIMIT}')
        sp = K.spheres_tensor(rec, self.device)
        if len(flat):
            # The capacity comes from the particles themselves, so the
            # coefficient kernel can fail only on invalid parameters:
            # checked here on the host, which spares homogeneous spheres
            # a device round trip before the field launch.
            plain = not any(K.is_layered(p) for p in flat)
            if plain:
                v = rec.view(np.float64).reshape(-1, 6)
                if not (np.isfinite(v).all() and (rec['a_p'] > 0.).all()):
                    raise ValueError('particle parameters must be finite '
                                     'with a_p > 0')
            ab, dab, nmax = K.particle_ab(flat, sp, inst.n_m,
                                          inst.wavelength, cap, deriv,
                                          check=not plain)
        else:
            ab = torch.zeros((1, 2, 2, 2), dtype=torch.float64,
                             device=self.device)
            dab, nmax = None, torch.zeros(1, dtype=torch.int32,
                                          device=self.device)
        return sp, item_start, ab, dab, nmax, cap

    def _aberration(self):
        '''Coefficient of a spherical-aberration phase applied to every
        particle's field (0: ideal optics; see theory/Aberrated.py).'''
        return 0.

    def _field_items(self, particle_lists, cartesian, bohren):
        sp, item_start, ab, _, nmax, cap = self._prepare(particle_lists)
        return K.field(self._coords, sp, item_start, ab, nmax, cap,
                       self.instrument.wavenumber(), cartesian, bohren,
                       self.double_precision, self._aberration())

    def _hologram_items(self, particle_lists, cartesian, bohren):
        sp, item_start, ab, _, nmax, cap = self._prepare(particle_lists)
        return K.hologram(self._coords, sp, item_start, ab, nmax, cap,
                          self.instrument.wavenumber(), cartesian, bohren,
                          self.double_precision, self._aberration())

    # ------------------------------------------------------------------
    def field(self, cartesian=True, bohren=True, device=False):
        '''Scattered field (3, npts) of all particles (superposed).'''
        f = self._field_items([list(self.particle)], cartesian, bohren)[0]
        if device:
            return f
        return K.to_numpy(f, torch.complex128)

    def scattered_field(self, particle, cartesian=True, bohren=True,
                        device=False):
        '''Field of one particle including exp(-i k z_p).'''
        f = self._field_items([[particle]], cartesian, bohren)[0]
        if device:
            return f
        return K.to_numpy(f, torch.complex128)

    def hologram(self, cartesian=True, bohren=True, device=False):
        '''Hologram |E + x|^2, numpy float64 (npts,) unless device=True.'''
        h = self._hologram_items([list(self.particle)], cartesian, bohren)[0]
        if device:
            return h
        return K.to_numpy(h, torch.float64)

    def batch_field(self, particle_lists, cartesian=True, bohren=True):
        '''(B, 3, npts) complex tensor, one particle list per item.'''
        B = len(particle_lists)
        npts = self._coordinates.shape[1]
        if B == 0 or max((len(pl) for pl in particle_lists), default=0) == 0:
            dt = torch.complex128 if self.double_precision else torch.complex64
            return torch.zeros((B, 3, npts), dtype=dt, device=self.device)
        return self._field_items([list(pl) for pl in particle_lists],
                                 cartesian, bohren)

    def batch_hologram(self, particle_lists, cartesian=True, bohren=True,
                       device=False):
        '''(B, npts) holograms, numpy float64 unless device=True.'''
        B = len(particle_lists)
        npts = self._coordinates.shape[1]
        if B == 0:
            h = torch.zeros((0, npts), dtype=torch.float64,
                            device=self.device)
        else:
            h = self._hologram_items([list(pl) for pl in particle_lists],
                                     cartesian, bohren)
        if device:
            return h
        return K.to_numpy(h, torch.float64)

    # ------------------------------------------------------------------
    def jac(self, device=False):
        '''dH/dp for p in x_p, y_p, z_p, a_p, n_p, k_p at the current state:
        dict name -> (npts,) float64.  Single sphere only, like the
        reference's jac (theory/jaxLorenzMie.py:373-374).'''
        if not isinstance(self.particle, Sphere) and not (
                hasattr(self.particle, 'a_p') and len(self.particle) == 1):
            raise TypeError('jac() supports single Sphere particles only')
        sp, _, ab, dab, nmax, cap = self._prepare([[self.particle]],
                                                  deriv=True)
        _, J = K.jacobian(self._coords, sp, ab, dab, nmax, cap,
                          self.instrument.wavenumber(),
                          aberration=self._aberration())
        J = J[0]
        if device:
            return {k: J[i] for i, k in enumerate(JAC_KEYS)}
        J = K.to_numpy(J, torch.float64)
        return {k: J[i] for i, k in enumerate(JAC_KEYS)}

    def hologram_and_jac(self, bohren=True):
        '''Hologram (npts,) and Jacobian (6, npts) tensors in one pass.'''
        sp, _, ab, dab, nmax, cap = self._prepare([[self.particle]],
                                                  deriv=True)
        h, J = K.jacobian(self._coords, sp, ab, dab, nmax, cap,
                          self.instrument.wavenumber(), bohren,
                          aberration=self._aberration())
        return h[0], J[0]
