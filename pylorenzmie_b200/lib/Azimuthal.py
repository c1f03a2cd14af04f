'''Azimuthal average of an image about a point (same contract as
lib/Azimuthal.py:avg): integer-radius bins, radius r = floor(hypot(x - x_p,
y - y_p)) in pixels, mean of the pixels in each bin from r = 0 outward.'''
import numpy as np


def avg(data, center=None):
    '''Azimuthal average of a 2-D image about center (x, y) (default: the
    image centre, (nx/2, ny/2)).'''
    data = np.asarray(data)
    ny, nx = data.shape
    x_p, y_p = (nx / 2., ny / 2.) if center is None else center
    r = np.hypot.outer(np.arange(ny) - float(y_p),
                       np.arange(nx) - float(x_p)).astype(np.int32).ravel()
    return np.bincount(r, data.ravel()) / np.bincount(r)
