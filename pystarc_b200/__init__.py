"""B200-native batched rigid-body Brownian-dynamics engine with PySTARC's entry points."""

__version__ = "0.1.0"
