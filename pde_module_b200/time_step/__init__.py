from .forwardEuler import ForwardEuler
from .heat import HeatRollout
from .fractional_step import FractionalStepLDC
from .wave import WaveSolver, wave_rollout
from .batched import BatchedHeatRollout, BatchedWaveRollout
