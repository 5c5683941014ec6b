from .ExplicitUniformGridStencil import ExplicitUniformGridStencil
from .laplacian import Laplacian
from .grad import Grad
from .divergence import Divergence
