from .functional_boundary import GridBoundary, FunctionBC, get_unique_key
from .immersed_boundary import ImmersedBoundary
from .boundary_functions import get_constant_func, get_ramp_func, BCFunction
from .flags import DIRICHLET, VON_NEUMANN, NO_BC, BC_SRING
