'''Abstract base of the parameter estimators (same contract as
analysis/BaseEstimator.py).'''
from abc import abstractmethod

from ..lib import LMObject


class BaseEstimator(LMObject):
    '''Estimators implement ``estimate(hologram) -> pandas.Series``.'''

    @abstractmethod
    def estimate(self, hologram):
        '''Estimate particle parameters from a normalized hologram.'''
