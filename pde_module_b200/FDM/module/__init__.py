from .ExplicitUniformGridStencil import ExplicitUniformGridStencil
from .laplacian import Laplacian
from .grad import Grad
from .divergence import Divergence
from .elementWiseOps import OuterProduct, scalarVectorMult
from .absorbing_layers import FarField, ViscousDampingLayer
