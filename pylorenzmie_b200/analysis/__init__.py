from .Hologram import Hologram
from .Mask import Mask
from .Optimizer import Optimizer

__all__ = ['Hologram', 'Mask', 'Optimizer']
