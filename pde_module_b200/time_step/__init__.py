from .forwardEuler import ForwardEuler
from .heat import HeatRollout
