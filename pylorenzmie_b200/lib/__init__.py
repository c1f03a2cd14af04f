from .meshgrid import meshgrid
from . import Azimuthal
from .LMObject import LMObject
from .lmtypes import (Property, Properties, Image, Images, Coordinates,
                      Coefficients, Field, Result, Results)

__all__ = ['meshgrid', 'Azimuthal', 'LMObject', 'Property', 'Properties', 'Image',
           'Images', 'Coordinates', 'Coefficients', 'Field', 'Result',
           'Results']
