'''Pixel coordinate grid (same contract as lib/meshgrid.py:10-40).'''
import numpy as np


def meshgrid(shape, corner=(0., 0.), flatten=True, dtype=float):
    '''(2, ny*nx) pixel coordinates, x row first; (2, ny, nx) if not flat.'''
    ny, nx = shape
    left, top = corner
    x = np.arange(left, left + nx, dtype=dtype)
    y = np.arange(top, top + ny, dtype=dtype)
    xy = np.array(np.meshgrid(x, y))
    return xy.reshape((2, -1)) if flatten else xy
