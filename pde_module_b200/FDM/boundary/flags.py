"""Boundary-condition flags (reference: FDM/boundary/flags.py:8-29)."""
NO_BC = 0
DIRICHLET = 1
VON_NEUMANN = 2
BC_SRING = {1: "DIRICHLET", 2: "VON_NEUMANN"}
FLUID_CELL = 0
SOLID_CELL = 1
