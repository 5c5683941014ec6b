from .forwardEuler import ForwardEuler
from .heat import HeatRollout, HeatSolver, heat_rollout
from .fractional_step import FractionalStepLDC, SlabFractionalStepLDC
from .wave import WaveSolver, wave_rollout
from .batched import BatchedHeatRollout, BatchedWaveRollout
from .rungeKatta import RungeKatta1, RungeKatta2, SignatureMismatchError
from .weakly_compressible import WeaklyCompressibleRK2, lid_driven_cavity_wc
