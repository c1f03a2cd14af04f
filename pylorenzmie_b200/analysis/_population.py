'''Objective of a differential-evolution search over a whole population in
one launch (lmb_chi2_batch): the batched form of the reference's per-
candidate objectives (analysis/DEEstimator.py:23-37,
analysis/RadialEstimator.py:17-37), which evaluate model.hologram() once per
candidate, in worker processes.'''
import numpy as np
import torch

from ..theory import _kernels as K

SPHERE_KEYS = ('x_p', 'y_p', 'z_p', 'a_p', 'n_p', 'k_p')


def batchable(model, variables):
    '''True when every searched variable is a parameter of a single
    homogeneous sphere (the population then goes to the GPU in one call).'''
    p = model.particle
    if isinstance(p, (list, tuple)) or K.is_layered(p) or not hasattr(p, 'a_p'):
        return False
    if len(p) != 1 or getattr(model, '_aberration', lambda: 0.)() != 0.:
        return False
    return all(v in SPHERE_KEYS for v in variables)


class PopulationChi2:
    '''callable(x) for scipy.optimize.differential_evolution with
    vectorized=True: x is (nvar, S) (or (nvar,)); returns the S values of
    sum(((H - data)/noise)^2), NaN residuals skipped.'''

    def __init__(self, model, data, coords, variables, noise):
        self.model = model
        dev = model.device
        c = np.atleast_2d(np.asarray(coords, dtype=float))
        c3 = np.zeros((3, c.shape[1]))
        c3[:c.shape[0]] = c
        self.coords = torch.from_numpy(c3).to(dev)
        self.data = torch.from_numpy(
            np.ascontiguousarray(data, dtype=np.float64)).to(dev)
        p = model.particle
        r = np.asarray(p.r_p, float) + np.asarray(
            getattr(p, 'r_0', (0., 0., 0.)), float)
        self.base = np.array([r[0], r[1], r[2], p.a_p, p.n_p,
                              getattr(p, 'k_p', 0.)])
        self.slots = [SPHERE_KEYS.index(v) for v in variables]
        inst = model.instrument
        self.n_m, self.wavelength = inst.n_m, inst.wavelength
        self.k = inst.wavenumber()
        self.noise = float(noise)
        self.fp64 = bool(getattr(model, 'double_precision', False))
        self.evaluations = 0

    def __call__(self, x):
        x = np.asarray(x, dtype=float)
        single = x.ndim == 1
        X = x.reshape(len(self.slots), -1)
        S = X.shape[1]
        P = np.tile(self.base, (S, 1))
        P[:, self.slots] = X.T
        rec = np.zeros(S, dtype=K.SPHERE_DTYPE)
        for j, key in enumerate(SPHERE_KEYS):
            rec[key] = P[:, j]
        dev = self.coords.device
        sp = K.spheres_tensor(rec, dev)
        cap = K.nmax_cap_for(P[:, 3], P[:, 4], P[:, 5], self.n_m,
                             self.wavelength)
        ab, _, nmax = K.sphere_ab(sp, self.n_m, self.wavelength, cap,
                                  check=False)
        item_start = torch.arange(S + 1, dtype=torch.int32, device=dev)
        chi2, bad = K.chi2(self.coords, self.data, self.noise, sp, item_start,
                           ab, nmax, cap, self.k, fp64=self.fp64,
                           nonfinite=True)
        chi2 = chi2.cpu().numpy()
        redo = np.flatnonzero(bad.cpu().numpy()) if not self.fp64 else []
        if len(redo):
            # candidates whose focal plane cuts the sphere: the partial
            # waves outgrow FP32's range there; FP64, as the reference
            sel = torch.from_numpy(redo).to(dev)
            n = len(redo)
            chi2[redo] = K.chi2(
                self.coords, self.data, self.noise, sp[sel],
                torch.arange(n + 1, dtype=torch.int32, device=dev),
                ab[sel], nmax[sel], cap, self.k, fp64=True).cpu().numpy()
        self.evaluations += S
        return float(chi2[0]) if single else chi2
