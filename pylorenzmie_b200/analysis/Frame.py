'''Full-frame analysis: features as crops of one camera frame, fitted
together (same contract as analysis/Frame.py).

``optimize`` replaces the reference's loop over features
(analysis/Frame.py:163-174, one scipy fit after another) by one batched
device fit of every feature that the device fit covers (grouped by free
variables, settings and layer count), streamed as optimize_batch is;
features it does not cover keep their own Optimizer.optimize.  Each
feature's optimizer is left holding its own result, as after
feature.optimize().  Detection needs a localizer object with
``localize(image) -> DataFrame`` of bbox, x_p, y_p rows
(analysis/Localizer.py, whose trackpy backend is not part of this
package); features can also be set from bounding boxes.
'''
import numpy as np
import pandas as pd

from ..lib import meshgrid
from ..theory.Instrument import Instrument
from ..theory.LorenzMie import LorenzMie
from .Hologram import Hologram
from .Feature import Feature
from .DEEstimator import estimate_many
from . import _fit
from ._fit import PARAM_KEYS


def _result_table(n, tables):
    '''DataFrame of n features' Optimizer.result rows (variables with their
    uncertainties, success, npix, redchi) from the batched groups' arrays;
    the same values and column types as pd.DataFrame of the Series.'''
    variables = tables[0][1]
    nv = len(variables)
    x, dp = np.empty((n, nv)), np.empty((n, nv))
    success = np.empty(n, dtype=bool)
    npix = np.empty(n, dtype=np.int64)
    redchi = np.empty(n)
    for idx, _, xs, ds, ss, ns, rs in tables:
        x[idx], dp[idx], success[idx], npix[idx], redchi[idx] = \
            xs, ds, ss, ns, rs
    cols = {}
    for j, v in enumerate(variables):
        cols[v] = x[:, j]
        cols['d' + v] = dp[:, j]
    cols['success'] = success
    cols['npix'] = npix
    cols['redchi'] = redchi
    return pd.DataFrame(cols)


class Frame(Hologram):
    '''Full-frame holographic microscopy analysis pipeline.'''

    def __init__(self, data=None, corner=(0., 0.), instrument=None,
                 localizer=None):
        self.instrument = instrument or Instrument()
        self.localizer = localizer
        self._features = []
        self._bboxes = []
        self._results = pd.DataFrame()
        self.corner = corner
        self._coordinates = None
        self._data = None
        if data is not None:
            self.data = data

    @property
    def data(self):
        return self._data

    @data.setter
    def data(self, data):
        self._features = []
        self._results = pd.DataFrame()
        self._data = data
        if data is not None:
            self._coordinates = meshgrid(data.shape, corner=self.corner,
                                         flatten=False)
        else:
            self._coordinates = None

    @property
    def shape(self):
        return (0, 0) if self._data is None else self._data.shape

    @property
    def is_grid(self):
        return True

    @property
    def results(self):
        return self._results

    @property
    def features(self):
        return self._features

    @property
    def bboxes(self):
        return self._bboxes

    @bboxes.setter
    def bboxes(self, bboxes):
        if (isinstance(bboxes, tuple) and len(bboxes) == 3
                and isinstance(bboxes[0], tuple)):
            bboxes = [bboxes]
        self._bboxes = list(bboxes)
        self._features = []
        for (x0, y0), w, h in self._bboxes:
            dim = min(w, h)
            feature = self[y0:y0 + dim, x0:x0 + dim]
            feature.particle.x_p = x0 + dim / 2.
            feature.particle.y_p = y0 + dim / 2.
            self._features.append(feature)

    def __getitem__(self, key):
        '''A Feature crop with the matching corner and the shared
        instrument.'''
        return Feature(Hologram.__getitem__(self, key),
                       model=LorenzMie(instrument=self.instrument))

    def detect(self):
        '''Detect and localize features (needs a localizer).'''
        if self._data is None:
            self._features = []
            self._bboxes = []
            return 0
        if self.localizer is None:
            raise RuntimeError('Frame.detect needs a localizer with '
                               'localize(image) -> DataFrame(bbox, x_p, y_p)')
        df = self.localizer.localize(self._data)
        self._features = []
        self._bboxes = []
        for _, row in df.iterrows():
            (x0, y0), w, h = row.bbox
            dim = min(w, h)
            feature = self[y0:y0 + dim, x0:x0 + dim]
            feature.particle.x_p = row.x_p
            feature.particle.y_p = row.y_p
            self._features.append(feature)
            self._bboxes.append(row.bbox)
        return len(self._features)

    def estimate(self):
        '''Estimate parameters of every feature.  The features' searches
        run side by side: each generation of all of them is one population
        launch (estimate_many); estimators without that form run one by
        one.'''
        feats = self.features
        side = [f for f in feats if hasattr(f.estimator, 'search') and
                hasattr(f.estimator, 'accept')]
        rest = feats
        if len(side) > 1:
            estimate_many([f.estimator for f in side], side, series=False)
            rest = [f for f in feats if not any(f is g for g in side)]
        for f in rest:
            f.estimate()

    def optimize(self):
        '''Fit every feature; one batched device fit per group of
        compatible features.  Returns the results DataFrame, one row per
        feature in order.'''
        feats = self.features
        groups = {}
        for i, f in enumerate(feats):
            opt = f.optimizer
            if not opt._device_fit_ok():
                continue
            part = f.model.particle
            layers = _fit.layers_of([part])
            inst = f.model.instrument
            key = (tuple(opt.variables),
                   tuple(sorted((k, repr(v)) for k, v in opt.settings.items())),
                   tuple(sorted(inst.properties.items())),
                   None if layers is None else layers[0],
                   str(f.model.device), opt._aberration())
            groups.setdefault(key, []).append(i)
        done = set()
        tables = []   # per group: the columns of Optimizer.result
        for key, idx in groups.items():
            members = [feats[i] for i in idx]
            opt0 = members[0].optimizer
            items = [f.optimizer._pixels(f) for f in members]
            starts = np.concatenate([f.optimizer._start() for f in members])
            layers = _fit.layers_of([f.model.particle for f in members])
            params, res, _ = _fit.fit_items(
                items, starts, members[0].model.instrument, opt0.variables,
                opt0.settings, device=members[0].model.device, layers=layers,
                autotune=len(members) >= 64, aberration=opt0._aberration())
            for j, f in enumerate(members):
                f.optimizer._data = np.asarray(items[j][0])
                f.optimizer.model.coordinates = items[j][2] if \
                    items[j][2] is not None else f.flat_coordinates
                f.optimizer._accept(params[j], res[j])
            done.update(idx)
            cols = [PARAM_KEYS.index(v) for v in opt0.variables]
            tables.append((idx, tuple(opt0.variables), params[:, cols],
                           res['dparams'][:, cols],
                           res['success'].astype(bool),
                           np.array([np.asarray(it[0]).size for it in items]),
                           res['redchi'].astype(float)))
        if len(done) == len(feats) and len({t[1] for t in tables}) == 1:
            # every feature fitted on the device with one variable list:
            # the table of their result Series, built from the arrays
            self._results = _result_table(len(feats), tables)
            return self._results
        results = []
        for i, f in enumerate(feats):
            if i not in done:
                f.optimize()
            results.append(f.optimizer.result)
        self._results = pd.DataFrame(results)
        return self._results

    def analyze(self, data=None):
        '''Detect, estimate and optimize.'''
        self.data = data
        self.detect()
        self.estimate()
        return self.optimize()
