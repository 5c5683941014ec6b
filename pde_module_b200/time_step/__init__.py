from .forwardEuler import ForwardEuler
from .heat import HeatRollout
from .fractional_step import FractionalStepLDC
