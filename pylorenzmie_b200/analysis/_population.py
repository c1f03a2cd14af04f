'''Objective of a differential-evolution search over a whole population in
one launch (lmb_chi2_batch): the batched form of the reference's per-
candidate objectives (analysis/DEEstimator.py:23-37,
analysis/RadialEstimator.py:17-37), which evaluate model.hologram() once per
candidate, in worker processes.

The searches of many features (Frame.estimate, analysis/Frame.py:158-161,
runs them one after another) go further: ``lockstep_de`` runs scipy's
differential_evolution for each on a thread of its own, and every
generation of all of them is evaluated together by ``CropPopulations`` in
one lmb_chi2_crops launch.  Each search keeps scipy's own code and random
stream, and each candidate's value is bit-identical to the one-search
launch, so a seeded search ends where it ends alone.'''
import threading

import numpy as np
import torch
from scipy.optimize import differential_evolution

from .. import _native
from .._device import ptr, stream_handle
from ..theory import _kernels as K

SPHERE_KEYS = ('x_p', 'y_p', 'z_p', 'a_p', 'n_p', 'k_p')
MAX_ITEMS = 65535          # candidates per launch (the grid's y extent)


def batchable(model, variables):
    '''True when every searched variable is a parameter of a single
    homogeneous sphere (the population then goes to the GPU in one call;
    an aberrated model's phase is applied in the same launch).'''
    p = model.particle
    if isinstance(p, (list, tuple)) or K.is_layered(p) or not hasattr(p, 'a_p'):
        return False
    if len(p) != 1:
        return False
    return all(v in SPHERE_KEYS for v in variables)


def aberration(model):
    '''Spherical-aberration coefficient c of a model (0: ideal optics).'''
    return float(getattr(model, '_aberration', lambda: 0.)())


def de_settings(settings):
    '''scipy settings of a population search: one objective call per
    generation (vectorized, deferred updating, as the reference's
    'deferred'); the reference's worker processes have no role here.'''
    settings = dict(settings)
    settings.pop('workers', None)
    settings['updating'] = 'deferred'
    settings['vectorized'] = True
    return settings


def _coords3(coords):
    c = np.atleast_2d(np.asarray(coords, dtype=float))
    c3 = np.zeros((3, c.shape[1]))
    c3[:c.shape[0]] = c
    return c3


def _records(P):
    rec = np.zeros(len(P), dtype=K.SPHERE_DTYPE)
    for j, key in enumerate(SPHERE_KEYS):
        rec[key] = P[:, j]
    return rec


class _Candidates:
    '''The fixed sphere parameters of one search and the slots its
    variables fill: candidates(x) -> (S, 6) sphere parameters.'''

    def __init__(self, model, variables):
        p = model.particle
        r = np.asarray(p.r_p, float) + np.asarray(
            getattr(p, 'r_0', (0., 0., 0.)), float)
        self.base = np.array([r[0], r[1], r[2], p.a_p, p.n_p,
                              getattr(p, 'k_p', 0.)])
        self.slots = [SPHERE_KEYS.index(v) for v in variables]

    def __call__(self, x):
        X = np.asarray(x, dtype=float).reshape(len(self.slots), -1)
        P = np.tile(self.base, (X.shape[1], 1))
        P[:, self.slots] = X.T
        return P


class PopulationChi2:
    '''callable(x) for scipy.optimize.differential_evolution with
    vectorized=True: x is (nvar, S) (or (nvar,)); returns the S values of
    sum(((H - data)/noise)^2), NaN residuals skipped.'''

    def __init__(self, model, data, coords, variables, noise):
        self.model = model
        dev = model.device
        self.coords = torch.from_numpy(_coords3(coords)).to(dev)
        self.data = torch.from_numpy(
            np.ascontiguousarray(data, dtype=np.float64)).to(dev)
        self.candidates = _Candidates(model, variables)
        inst = model.instrument
        self.n_m, self.wavelength = inst.n_m, inst.wavelength
        self.k = inst.wavenumber()
        self.noise = float(noise)
        self.fp64 = bool(getattr(model, 'double_precision', False))
        self.aberr = aberration(model)
        self.evaluations = 0

    def _chi2(self, sp, ab, nmax, cap, fp64):
        '''(chi2, nonfinite) of candidates sp; aberrated models through
        lmb_chi2_crops with the whole pixel set as the one crop.'''
        dev = self.coords.device
        S = sp.shape[0]
        item_start = torch.arange(S + 1, dtype=torch.int32, device=dev)
        if not self.aberr:
            return K.chi2(self.coords, self.data, self.noise, sp, item_start,
                          ab, nmax, cap, self.k, fp64=fp64, nonfinite=True)
        n = self.coords.shape[1]
        crop_start = torch.tensor([0, n], dtype=torch.int64, device=dev)
        item_crop = torch.zeros(S, dtype=torch.int32, device=dev)
        return K.chi2_crops(self.coords, self.data, self.noise, crop_start,
                            item_crop, n, sp, item_start, ab, nmax, cap,
                            self.k, fp64=fp64, aberration=self.aberr)

    def __call__(self, x):
        x = np.asarray(x, dtype=float)
        single = x.ndim == 1
        P = self.candidates(x)
        S = len(P)
        dev = self.coords.device
        sp = K.spheres_tensor(_records(P), dev)
        cap = K.nmax_cap_for(P[:, 3], P[:, 4], P[:, 5], self.n_m,
                             self.wavelength)
        ab, _, nmax = K.sphere_ab(sp, self.n_m, self.wavelength, cap,
                                  check=False)
        chi2, bad = self._chi2(sp, ab, nmax, cap, self.fp64)
        chi2 = chi2.cpu().numpy()
        redo = np.flatnonzero(bad.cpu().numpy()) if not self.fp64 else []
        if len(redo):
            # candidates whose focal plane cuts the sphere: the partial
            # waves outgrow FP32's range there; FP64, as the reference
            sel = torch.from_numpy(redo).to(dev)
            chi2[redo] = self._chi2(sp[sel], ab[sel], nmax[sel], cap,
                                    True)[0].cpu().numpy()
        self.evaluations += S
        return float(chi2[0]) if single else chi2


class CropPopulations:
    '''The objectives of several searches, each over a crop of its own,
    evaluated together: ``evaluate({search: x})`` computes every population
    it is given in one lmb_chi2_crops launch (per 65535 candidates).  The
    searches share the instrument, the noise and the precision.

    searches : list of (model, data, coords, variables), as PopulationChi2;
        the models share the instrument and the aberration.
    '''

    def __init__(self, searches, noise):
        model = searches[0][0]
        self.device = dev = model.device
        c3 = [_coords3(c) for _, _, c, _ in searches]
        sizes = [c.shape[1] for c in c3]
        self.coords = torch.from_numpy(
            np.ascontiguousarray(np.hstack(c3))).to(dev)
        self.data = torch.from_numpy(np.concatenate(
            [np.asarray(d, dtype=np.float64).ravel() for _, d, _, _ in searches]
        )).to(dev)
        self.crop_start = torch.from_numpy(np.concatenate(
            [[0], np.cumsum(sizes)]).astype(np.int64)).to(dev)
        self.max_npts = max(sizes)
        self.candidates = [_Candidates(m, v) for m, _, _, v in searches]
        inst = model.instrument
        self.n_m, self.wavelength = inst.n_m, inst.wavelength
        self.k = inst.wavenumber()
        self.noise = float(noise)
        self.fp64 = bool(getattr(model, 'double_precision', False))
        self.aberr = aberration(model)
        self.evaluations = 0

    def evaluate(self, batch):
        '''batch: {search index: x}, x as scipy passes it ((nvar, S), or
        (nvar,) for one candidate); returns {search index: values}.'''
        order = sorted(batch)
        P = [self.candidates[i](batch[i]) for i in order]
        counts = [len(p) for p in P]
        crop = np.concatenate([np.full(n, i, dtype=np.int32)
                               for i, n in zip(order, counts)])
        P = np.vstack(P)
        chi2 = np.empty(len(P))
        for a in range(0, len(P), MAX_ITEMS):
            b = min(a + MAX_ITEMS, len(P))
            chi2[a:b] = self._launch(P[a:b], crop[a:b])
        self.evaluations += len(P)
        out, at = {}, 0
        for i, n in zip(order, counts):
            v = chi2[at:at + n]
            at += n
            out[i] = float(v[0]) if np.ndim(batch[i]) == 1 else v
        return out

    def _buffers(self, n, cap):
        '''Pinned staging and device buffers for n candidates of up to cap
        orders, kept between generations and grown when needed (a
        generation ends with its results read back, so the next one may
        reuse them).'''
        b = getattr(self, '_bufs', None)
        if b is None or b['n'] < n or b['cap'] < cap:
            n = max(n, b['n'] if b else 0)
            cap = max(cap, b['cap'] if b else 0)
            dev = self.device
            lib = _native.load()
            ws = lib.lmb_chi2_workspace_bytes(int(self.max_npts), n)
            b = dict(n=n, cap=cap, ws_bytes=ws,
                     host_in=torch.empty(n * 52, dtype=torch.uint8,
                                         pin_memory=True),
                     dev_in=torch.empty(n * 52, dtype=torch.uint8,
                                        device=dev),
                     host_out=torch.empty(n * 12, dtype=torch.uint8,
                                          pin_memory=True),
                     item_start=torch.arange(n + 1, dtype=torch.int32,
                                             device=dev),
                     ab=torch.empty(n * (cap + 1) * 4, dtype=torch.float64,
                                    device=dev),
                     nmax=torch.empty(n, dtype=torch.int32, device=dev),
                     status=torch.empty(n, dtype=torch.int32, device=dev),
                     chi2=torch.empty(n, dtype=torch.float64, device=dev),
                     bad=torch.empty(n, dtype=torch.int32, device=dev),
                     ws=torch.empty(max(ws, 1), dtype=torch.uint8,
                                    device=dev))
            self._bufs = b
        return b

    def _launch(self, P, crop):
        '''chi^2 of candidates P (n, 6) against their crops: the sphere
        records and crop indices in one copy from pinned memory, the
        coefficients and sums into kept buffers (lmb_sphere_ab,
        lmb_chi2_crops), the sums and overflow counts read back together;
        FP32 sums that overflowed are redone in FP64.'''
        dev = self.device
        n = len(P)
        cap = K.nmax_cap_for(P[:, 3], P[:, 4], P[:, 5], self.n_m,
                             self.wavelength)
        b = self._buffers(n, cap)
        hin = b['host_in'].numpy()
        hin[:48 * n].view(np.float64)[:] = np.ascontiguousarray(
            P, dtype=np.float64).ravel()
        hin[48 * n:52 * n].view(np.int32)[:] = crop
        b['dev_in'][:52 * n].copy_(b['host_in'][:52 * n], non_blocking=True)
        sp = b['dev_in'][:48 * n].view(torch.float64).view(n, 6)
        item_crop = b['dev_in'][48 * n:52 * n].view(torch.int32)
        ab = b['ab'][:n * (cap + 1) * 4].view(n, cap + 1, 2, 2)
        nmax = b['nmax'][:n]
        lib = _native.load()
        stream = stream_handle(dev)
        _native.check(lib.lmb_sphere_ab(
            ptr(sp), n, float(self.n_m), float(self.wavelength), cap, ptr(ab),
            None, ptr(nmax), ptr(b['status']), stream), 'lmb_sphere_ab')
        _native.check(lib.lmb_chi2_crops(
            ptr(self.coords), self.coords.shape[1], ptr(self.data),
            float(self.noise), ptr(self.crop_start),
            self.crop_start.shape[0] - 1, ptr(item_crop), int(self.max_npts),
            ptr(sp), ptr(b['item_start']), n, ptr(ab), ptr(nmax), cap,
            float(self.k), K._flags(True, True, self.fp64), ptr(b['chi2']),
            ptr(b['bad']), ptr(b['ws']), b['ws_bytes'], stream,
            float(self.aberr)), 'lmb_chi2_crops')
        hout = b['host_out']
        hout[:8 * n].view(torch.float64).copy_(b['chi2'][:n],
                                               non_blocking=True)
        hout[8 * n:12 * n].view(torch.int32).copy_(b['bad'][:n],
                                                   non_blocking=True)
        torch.cuda.current_stream(dev).synchronize()
        out = hout.numpy()
        chi2 = out[:8 * n].view(np.float64).copy()
        bad = out[8 * n:12 * n].view(np.int32).copy()
        redo = np.flatnonzero(bad) if not self.fp64 else []
        if len(redo):
            # FP32 overflow where the focal plane cuts the sphere: FP64
            sel = torch.from_numpy(redo).to(dev)
            m = len(redo)
            chi2[redo] = K.chi2_crops(
                self.coords, self.data, self.noise, self.crop_start,
                item_crop[sel], self.max_npts, sp[sel],
                torch.arange(m + 1, dtype=torch.int32, device=dev), ab[sel],
                nmax[sel], cap, self.k, fp64=True,
                aberration=self.aberr)[0].cpu().numpy()
        return chi2


class _Aborted(Exception):
    '''Ends a search whose companions failed.'''


class Lockstep:
    '''Gathers one objective call from every running search and evaluates
    them together.  ``workers`` threads take part; each runs one search at a
    time and calls ``leave()`` when it has no more.  A generation runs when
    every live worker has submitted, on the thread that completed it, under
    ``device`` and ``stream`` (the caller's; worker threads start on the
    default device and stream).'''

    def __init__(self, workers, evaluate, device=None, stream=None):
        self._cv = threading.Condition()
        self._live = workers
        self._pending = {}
        self._results = {}
        self.error = None
        self._evaluate = evaluate
        self._device, self._stream = device, stream
        self.generations = 0

    def objective(self, i):
        return lambda x: self._submit(i, x)

    def _submit(self, i, x):
        with self._cv:
            if self.error is not None:
                raise _Aborted()
            self._pending[i] = x
            if len(self._pending) == self._live:
                self._run()
            while i not in self._results and self.error is None:
                self._cv.wait(1.0)
            if i in self._results:
                return self._results.pop(i)
            raise _Aborted()

    def leave(self):
        with self._cv:
            self._live -= 1
            if self._pending and len(self._pending) == self._live:
                self._run()

    def fail(self, error):
        with self._cv:
            if self.error is None:
                self.error = error
            self._cv.notify_all()

    def _run(self):
        batch, self._pending = self._pending, {}
        if self.error is None:
            try:
                if self._device is None:
                    self._results.update(self._evaluate(batch))
                else:
                    with torch.cuda.device(self._device), \
                            torch.cuda.stream(self._stream):
                        self._results.update(self._evaluate(batch))
                self.generations += 1
            except BaseException as e:   # handed to every search
                self.error = e
        self._cv.notify_all()


def lockstep_de(problems, evaluate, workers=256, device=None, stream=None):
    '''scipy differential_evolution for each of ``problems`` (dicts with
    bounds, popsize, seed, settings), side by side: every generation's
    populations of all running searches go to ``evaluate`` together (see
    Lockstep).  Returns the OptimizeResults in order; an exception of any
    search or of ``evaluate`` is raised after every thread has ended.'''
    n = len(problems)
    results = [None] * n
    if n == 0:
        return results
    nw = max(1, min(n, int(workers)))
    step = Lockstep(nw, evaluate, device, stream)
    queue = iter(range(n))
    qlock = threading.Lock()

    def worker():
        try:
            while step.error is None:
                with qlock:
                    j = next(queue, None)
                if j is None:
                    break
                pr = problems[j]
                with np.errstate(over='ignore', invalid='ignore'):
                    results[j] = differential_evolution(
                        step.objective(j), pr['bounds'],
                        popsize=pr['popsize'], seed=pr['seed'],
                        **de_settings(pr['settings']))
        except _Aborted:
            pass
        except BaseException as e:
            step.fail(e)
        finally:
            step.leave()

    threads = [threading.Thread(target=worker, daemon=True)
               for _ in range(nw)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    if step.error is not None:
        raise step.error
    return results
