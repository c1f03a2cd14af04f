'''Base class with the reference's properties protocol (lib/LMObject.py).

``properties`` is both the serialization format and the optimizer's
parameter vector; JSON and pandas round trips keep the reference's format.
'''
import json
import logging
from abc import ABC, abstractmethod

import numpy as np
import pandas as pd

from .meshgrid import meshgrid


class LMObject(ABC):
    meshgrid = staticmethod(meshgrid)
    __hash__ = None

    @property
    def logger(self):
        return logging.getLogger(
            f'{self.__class__.__module__}.{self.__class__.__qualname__}')

    def __eq__(self, other):
        if not isinstance(other, self.__class__):
            return NotImplemented
        return self.properties == other.properties

    @property
    @abstractmethod
    def properties(self):
        return dict()

    @properties.setter
    def properties(self, properties):
        for name, value in properties.items():
            if hasattr(self, name):
                setattr(self, name, value)
            else:
                self.logger.debug('Ignoring unknown property: %s', name)

    def to_json(self, **kwargs):
        def np_encoder(obj):
            if isinstance(obj, np.generic):
                return obj.item()
        return json.dumps(self.properties, default=np_encoder, **kwargs)

    def from_json(self, s):
        self.properties = json.loads(s)

    def to_pandas(self, **kwargs):
        return pd.Series(self.properties, **kwargs)

    def from_pandas(self, series):
        self.properties = series.to_dict()
