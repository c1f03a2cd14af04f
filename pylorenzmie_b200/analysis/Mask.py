'''Random pixel subset for fitting (same contract as analysis/Mask.py).'''
import ctypes
from dataclasses import dataclass

import numpy as np

from .. import _native
from ..lib import LMObject


_MT_BLOCKS = None


def _mt_blocks_ok():
    '''Whether lmb_mask_select's MT19937 layout (the generator's words
    advanced by the library) reproduces its next_double layout on this
    numpy: the same subsets and the same final state over draws that
    straddle several blocks, checked once on scratch generators.'''
    global _MT_BLOCKS
    if _MT_BLOCKS is None:
        ok = True
        g = [np.random.MT19937(2024), np.random.MT19937(2024)]
        for n, frac in ((1, 0.5), (311, 0.1), (1247, 0.7), (5000, 0.3)):
            out = []
            for layout, bg in enumerate(g):
                idx = np.empty(n, dtype=np.int64)
                cnt = ctypes.c_longlong()
                st = _native.load().lmb_mask_select(
                    bg.ctypes.bit_generator.value, n, frac, None, layout,
                    idx.ctypes.data, ctypes.byref(cnt))
                ok = ok and st == _native.LMB_OK
                out.append(idx[:cnt.value])
            ok = ok and np.array_equal(out[0], out[1])
        s0, s1 = (bg.state['state'] for bg in g)
        ok = (ok and np.array_equal(s0['key'], s1['key'])
              and s0['pos'] == s1['pos'])
        _MT_BLOCKS = bool(ok)
    return _MT_BLOCKS


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
        layout = int(isinstance(bg, np.random.MT19937) and _mt_blocks_ok())
        with bg.lock:
            st = _native.load().lmb_mask_select(
                bg.ctypes.bit_generator.value, n, float(self.fraction),
                None if exclude is None else exclude.ctypes.data, layout,
                index.ctypes.data, ctypes.byref(count))
        _native.check(st, 'lmb_mask_select')
        self._index = index[:count.value]
        mask = np.zeros(n, dtype=bool)
        mask[self._index] = True
        self._mask = mask.reshape(shape)

    def apply(self, hologram):
        '''Selected pixel values (nsel,) and coordinates (2, nsel); a fresh
        random subset each call (analysis/Mask.py:82-105).  The pixels are
        gathered by index: a crop of a frame is a strided view, which a
        flattening copy would copy whole.'''
        self.shape = hologram.shape
        idx = self._index
        data = np.asarray(hologram.data)
        if data.ndim == 2:
            rows, cols = np.divmod(idx, data.shape[1])
            values = data[rows, cols]
            if getattr(hologram, 'is_grid', False):
                x0, y0 = hologram.corner
                coords = np.empty((2, idx.size))
                np.add(cols, float(x0), out=coords[0])
                np.add(rows, float(y0), out=coords[1])
            else:
                coords = hologram.coordinates[:, rows, cols]
            return values, coords
        return data.reshape(-1)[idx], hologram.flat_coordinates[:, idx]
