'''Differentiable holograms: torch.autograd.Function over the CUDA kernels.

``hologram(params, coordinates, instrument)`` returns the (B, npts) FP32
holograms of B single spheres, params (B, 6) = (x_p, y_p, z_p, a_p, n_p,
k_p).  Its backward pass is the hand-written VJP kernel
(``lmb_hologram_vjp``): it recomputes the Bessel and angular recurrences
pixel by pixel in forward mode and reduces g * dH/dparam over the pixels,
so nothing per order or per pixel is stored between forward and backward
(only the O(n_max) Mie coefficients and their parameter derivatives).
``jacobian`` returns the full per-pixel 6-column Jacobian instead.

No reference counterpart runs here: the reference torch backend is not
differentiable (theory/torchLorenzMie.py:293-300); its JAX backend's
jacfwd (theory/jaxLorenzMie.py:283-286) is the analogue.
'''
import numpy as np
import torch

from . import _kernels as K
from .Instrument import Instrument


def _prepare(params, instrument):
    p = params.detach().to(torch.float64).contiguous()
    inst = instrument or Instrument()
    host = p.cpu().numpy()
    cap = K.nmax_cap_for(host[:, 3], host[:, 4], host[:, 5], inst.n_m,
                         inst.wavelength)
    ab, dab, nmax = K.sphere_ab(p, inst.n_m, inst.wavelength, cap, deriv=True)
    return p, inst, cap, ab, dab, nmax


def _coords(coordinates, device):
    c = torch.as_tensor(coordinates, dtype=torch.float64, device=device)
    if c.shape[0] == 2:
        c = torch.cat([c, torch.zeros((1, c.shape[1]), dtype=torch.float64,
                                      device=device)])
    return c.contiguous()


class HologramFunction(torch.autograd.Function):
    '''H(params) with dH/dparams from the VJP kernel.'''

    @staticmethod
    def forward(ctx, params, coordinates, instrument, bohren):
        p, inst, cap, ab, dab, nmax = _prepare(params, instrument)
        B = p.shape[0]
        item_start = torch.arange(B + 1, dtype=torch.int32, device=p.device)
        h = K.hologram(coordinates, p, item_start, ab, nmax, cap,
                       inst.wavenumber(), True, bohren, False)
        ctx.save_for_backward(p, coordinates, ab, dab, nmax)
        ctx.inst, ctx.cap, ctx.bohren = inst, cap, bohren
        return h

    @staticmethod
    def backward(ctx, gout):
        p, coordinates, ab, dab, nmax = ctx.saved_tensors
        grad = K.hologram_vjp(coordinates, p, ab, dab, nmax, ctx.cap,
                              ctx.inst.wavenumber(), gout.contiguous(),
                              ctx.bohren)
        return grad.to(p.dtype), None, None, None


def hologram(params, coordinates, instrument=None, bohren=True):
    '''Differentiable (B, npts) float32 holograms of B spheres.'''
    if params.dim() == 1:
        params = params.unsqueeze(0)
    c = _coords(coordinates, params.device)
    return HologramFunction.apply(params, c, instrument, bohren)


def jacobian(params, coordinates, instrument=None, bohren=True):
    '''Holograms (B, npts) and Jacobians (B, 6, npts), float64 tensors.'''
    if params.dim() == 1:
        params = params.unsqueeze(0)
    p, inst, cap, ab, dab, nmax = _prepare(params, instrument)
    c = _coords(coordinates, p.device)
    return K.jacobian(c, p, ab, dab, nmax, cap, inst.wavenumber(), bohren)
