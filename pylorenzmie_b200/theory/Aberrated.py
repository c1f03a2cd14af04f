'''Lorenz-Mie model of an instrument with spherical aberration (same
contract as theory/Aberrated.py).

``Aberrated(base)`` returns a subclass of a LorenzMie model whose scattered
fields carry the phase exp(i Phi), Phi = (4 n_m^3 / k) s r^4/(r^2 + z_p^2)^2
(theory/Aberrated.py:41-79), s = ``spherical`` in wavelengths, k the
in-medium wave number (rad/pixel), r the in-plane distance from each
particle and z_p its axial position, both in pixels.  Here the phase is
applied inside the field kernel (lmb_field_aberrated /
lmb_hologram_aberrated), per particle and pixel, before the superposition.
The device fits include it (lmb_fit_batch_aberrated: the phase enters the
hologram and the x_p, y_p, z_p columns of the Jacobian): with ``spherical``
among an Optimizer's fixed parameters (a calibrated instrument), optimize,
optimize_batch and optimize_stream fit this model on the GPU.  With it free
-- the reference's default, whose fixed list does not name it -- the fit
runs through scipy's host loop on this model's holograms, as the
reference's does.  ``jac()`` includes the aberration
(lmb_jacobian_aberrated); ``spherical`` itself has no column, so a host
fit that frees it differentiates it numerically.
'''
from .LorenzMie import LorenzMie


def Aberrated(base_class):
    '''An aberrated subclass of a LorenzMie model class.'''

    class AberratedLorenzMie(base_class):

        def __init__(self, *args, spherical=0., **kwargs):
            super().__init__(*args, **kwargs)
            self.spherical = spherical

        @property
        def properties(self):
            return {**super().properties, 'spherical': self.spherical}

        @properties.setter
        def properties(self, properties):
            base_class.properties.fset(self, properties)


        def _aberration(self):
            if self.spherical == 0.:
                return 0.
            inst = self.instrument
            return 4. * inst.n_m ** 3 / inst.wavenumber() * self.spherical


    return AberratedLorenzMie


AberratedLorenzMie = Aberrated(LorenzMie)
# a module-level name, so that instances pickle
AberratedLorenzMie.__qualname__ = 'AberratedLorenzMie'
AberratedLorenzMie.__name__ = 'AberratedLorenzMie'
