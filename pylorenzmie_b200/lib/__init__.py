from .meshgrid import meshgrid
from .LMObject import LMObject
from .lmtypes import (Property, Properties, Image, Images, Coordinates,
                      Coefficients, Field, Result, Results)

__all__ = ['meshgrid', 'LMObject', 'Property', 'Properties', 'Image',
           'Images', 'Coordinates', 'Coefficients', 'Field', 'Result',
           'Results']
