"""Finite-difference operators on uniform grids (reference: FDM/__init__.py)."""
from .module import (Laplacian, Grad, Divergence, ExplicitUniformGridStencil, OuterProduct, scalarVectorMult,
                     FarField, ViscousDampingLayer)
from .boundary import GridBoundary, ImmersedBoundary
from . import kernel, functional, module, boundary
