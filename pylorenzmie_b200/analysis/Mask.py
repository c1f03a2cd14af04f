'''Random pixel subset for fitting (same contract as analysis/Mask.py).'''
import ctypes
from dataclasses import dataclass

import numpy as np

from .. import _native
from ..lib import LMObject


@dataclass
class Mask(LMObject):
    shape: tuple | None = None
    fraction: float = 0.1
    exclude: np.ndarray | None = None

    def __post_init__(self):
        self._mask = np.empty((0, 0), dtype=bool)
        self.update()

    def __setattr__(self, prop, value):
        super().__setattr__(prop, value)
        if prop in ('shape', 'fraction', 'exclude') and hasattr(self, '_mask'):
            self.update()

    def __call__(self):
        return self._mask

    @LMObject.properties.getter
    def properties(self):
        return dict(fraction=self.fraction)

    def update(self):
        '''Draw a fresh subset: np.random.rand(*shape) < fraction, without
        the excluded pixels (analysis/Mask.py:64-80), drawn by the library
        on the global generator's own bit generator (lmb_mask_select: the
        same draws, so the same subset and generator state as numpy's).'''
        if self.shape is None:
            return
        shape = tuple(int(v) for v in np.atleast_1d(self.shape))
        n = int(np.prod(shape))
        exclude = None
        if self.exclude is not None and np.shape(self.exclude) == shape:
            exclude = np.ascontiguousarray(self.exclude, dtype=np.uint8)
        index = np.empty(n, dtype=np.int64)
        count = ctypes.c_longlong()
        bg = np.random.mtrand._rand._bit_generator
        with bg.lock:
            st = _native.load().lmb_mask_select(
                bg.ctypes.bit_generator.value, n, float(self.fraction),
                None if exclude is None else exclude.ctypes.data,
                index.ctypes.data, ctypes.byref(count))
        _native.check(st, 'lmb_mask_select')
        self._index = index[:count.value]
        mask = np.zeros(n, dtype=bool)
        mask[self._index] = True
        self._mask = mask.reshape(shape)

    def apply(self, hologram):
        '''Selected pixel values (nsel,) and coordinates (2, nsel); a fresh
        random subset each call (analysis/Mask.py:82-105).'''
        self.shape = hologram.shape
        idx = self._index
        data = np.asarray(hologram.data).reshape(-1)[idx]
        return data, hologram.flat_coordinates[:, idx]
