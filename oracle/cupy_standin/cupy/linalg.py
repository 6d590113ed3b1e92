"""``cupy.linalg`` stand-in: NumPy's linalg (test infrastructure only)."""
from numpy.linalg import *  # noqa: F401,F403
