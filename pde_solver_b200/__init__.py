"""B200-native structured-grid solve path of pde_solver (libpdeb200.so + host API)."""
from . import abi
from .problem import FaceBC, GridProblem, default_options

__all__ = ["abi", "FaceBC", "GridProblem", "default_options"]
