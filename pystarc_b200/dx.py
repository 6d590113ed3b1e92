"""OpenDX scalar grids: the container the force engine uploads.

``DXGrid`` has the attributes the reference's ``DXGrid`` exposes to the batched
engine (pystarc/forces/electrostatic/grid_force.py:95-145): ``origin`` (3,),
``delta`` (3,3, orthogonal), ``data`` (nx,ny,nz) with z fastest (C order).
The reader accepts the same DX subset the reference parses; the writer emits
it.  Values are kept as float32 -- the engine's grid storage type -- unless the
caller passes float64 data.
"""

from __future__ import annotations

from pathlib import Path

import numpy as np


class DXGrid:
    def __init__(self, origin, delta, data):
        self.origin = np.asarray(origin, dtype=float)
        delta = np.asarray(delta, dtype=float)
        self.delta = np.diag(delta) if delta.ndim == 1 else delta
        self.data = np.asarray(data)
        self.shape = np.array(self.data.shape)

    @property
    def spacing(self) -> np.ndarray:
        return np.array([self.delta[i, i] for i in range(3)])

    @classmethod
    def from_file(cls, path, dtype=np.float32) -> "DXGrid":
        origin = np.zeros(3)
        delta = np.zeros((3, 3))
        shape = np.zeros(3, dtype=int)
        chunks = []
        with open(path) as fh:
            in_data = False
            row = 0
            for line in fh:
                line = line.strip()
                if not line or line.startswith("#"):
                    continue
                if line.startswith("object 1"):
                    parts = line.split()
                    shape[:] = int(parts[-3]), int(parts[-2]), int(parts[-1])
                elif line.startswith("origin"):
                    origin[:] = [float(v) for v in line.split()[1:4]]
                elif line.startswith("delta"):
                    delta[row] = [float(v) for v in line.split()[1:4]]
                    row += 1
                elif line.startswith("object 3"):
                    in_data = True
                elif in_data:
                    if line.startswith("object") or line.startswith("attribute"):
                        break
                    chunks.append(line)
        data = np.array(" ".join(chunks).split(), dtype=np.float64)
        if data.size != int(np.prod(shape)):
            raise ValueError(f"{path}: expected {int(np.prod(shape))} values, found {data.size}")
        if not np.all(np.isfinite(data)):
            raise ValueError(f"{path}: grid holds NaN or Inf values")
        return cls(origin, delta, data.reshape(tuple(shape)).astype(dtype))

    def write(self, path) -> None:
        nx, ny, nz = self.data.shape
        flat = np.asarray(self.data, dtype=np.float64).ravel()
        with open(Path(path), "w") as fh:
            fh.write(f"object 1 class gridpositions counts {nx} {ny} {nz}\n")
            fh.write("origin {:.6f} {:.6f} {:.6f}\n".format(*self.origin))
            for i in range(3):
                fh.write("delta {:.6f} {:.6f} {:.6f}\n".format(*self.delta[i]))
            fh.write(f"object 2 class gridconnections counts {nx} {ny} {nz}\n")
            fh.write(f"object 3 class array type double rank 0 items {flat.size} data follows\n")
            for i in range(0, flat.size, 3):
                fh.write(" ".join(f"{v:.9e}" for v in flat[i:i + 3]) + "\n")
            fh.write('object 4 class field\n')

    def __repr__(self):
        nx, ny, nz = self.data.shape
        return f"DXGrid({nx}x{ny}x{nz}, origin={self.origin}, spacing={self.spacing})"
