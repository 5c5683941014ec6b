from .stencil import Stencil, tuplify
from .hooks import setup, before_forward, after_forward
