from .forwardEuler import ForwardEuler
from .heat import HeatRollout, HeatSolver, heat_rollout
from .fractional_step import FractionalStepLDC, SlabFractionalStepLDC
from .wave import WaveSolver, wave_rollout
from .batched import BatchedHeatRollout, BatchedWaveRollout
from .rungeKatta import RungeKatta1, RungeKatta2, SignatureMismatchError
