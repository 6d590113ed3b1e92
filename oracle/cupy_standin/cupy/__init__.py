"""NumPy-backed stand-in for the ``cupy`` module (test infrastructure only).

It exists so that the reference's own ``GPUBatchForceEngine`` and
``GPUBatchSimulator`` (pystarc/forces/gpu_batch_engine.py,
pystarc/simulation/gpu_batch_simulator.py) run unchanged on a CPU when golden
fixtures are generated.  Every array operation those files use is NumPy's, which
CuPy mirrors.  The one CUDA kernel they launch, ``batch_force_kernel``
(gpu_batch_engine.py:65-123), is provided by ``RawKernel`` below as the oracle's
CPU restatement of that kernel (``oracle.forces.k1_batch_force``).

Nothing in the product imports this module.
"""

from __future__ import annotations

import numpy as _np
from numpy import *  # noqa: F401,F403  (array API surface the reference uses)

from . import linalg  # noqa: F401
from . import cuda  # noqa: F401

bool_ = _np.bool_
float64 = _np.float64
float32 = _np.float32
int32 = _np.int32
int64 = _np.int64
ndarray = _np.ndarray


def asnumpy(a):
    return _np.asarray(a)


def asarray(a, dtype=None):
    return _np.asarray(a, dtype=dtype)


class RawKernel:
    """Runs the named reference kernel through the oracle's CPU restatement."""

    def __init__(self, code: str, name: str):
        if name != "batch_force_kernel":
            raise NotImplementedError(f"stand-in has no restatement of {name}")
        self.name = name

    def __call__(self, grid, block, args):
        from oracle.forces import k1_batch_force_flat

        k1_batch_force_flat(*args)
