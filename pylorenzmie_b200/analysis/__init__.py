from .Hologram import Hologram
from .Mask import Mask
from .Optimizer import Optimizer
from .BaseEstimator import BaseEstimator
from .DEEstimator import DEEstimator
from .RadialEstimator import RadialEstimator
from .Feature import Feature
from .Frame import Frame

__all__ = ['Hologram', 'Mask', 'Optimizer', 'BaseEstimator', 'DEEstimator',
           'RadialEstimator', 'Feature', 'Frame']
