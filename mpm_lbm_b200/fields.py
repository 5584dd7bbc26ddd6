"""Field views that mimic the Taichi fields callers of the reference read.

Reference callers use ``field.to_numpy()`` / ``field.from_numpy()``,
``field[None]`` for scalars and ``field.shape``.  These views expose device
tensors held in the lattice layout (x fastest, planar components) in the
reference layout ((nx, ny, nz[, comps]) C order, z fastest).
"""

from __future__ import annotations

import numpy as np
import torch


def lattice_to_ref(t: torch.Tensor, dims, comps) -> torch.Tensor:
    """(comps, pitch) or (pitch,) lattice tensor -> (nx, ny, nz[, comps]) view."""
    nx, ny, nz = dims
    n = nx * ny * nz
    if comps:
        return t[..., :n].reshape(comps, nz, ny, nx).permute(3, 2, 1, 0)
    return t[:n].reshape(nz, ny, nx).permute(2, 1, 0)


def ref_to_lattice(a, dims, comps, out: torch.Tensor):
    """Write an (nx, ny, nz[, comps]) array into a lattice tensor."""
    nx, ny, nz = dims
    n = nx * ny * nz
    t = torch.as_tensor(np.ascontiguousarray(a)).to(out.device)
    if comps:
        flat = t.permute(3, 2, 1, 0).reshape(comps, n)
        out[:, :n] = flat.to(out.dtype)
    else:
        out[:n] = t.permute(2, 1, 0).reshape(n).to(out.dtype)


class CellField:
    """A lattice field in the reference's shape, backed by device tensors."""

    def __init__(self, dims, comps, np_dtype, get, put=None, name=""):
        self.dims = tuple(dims)
        self.comps = comps
        self.np_dtype = np.dtype(np_dtype)
        self._get = get
        self._put = put
        self.name = name

    @property
    def shape(self):
        return self.dims

    @property
    def n(self):
        return self.comps

    def to_torch(self) -> torch.Tensor:
        """Reference-shaped device view (no copy where possible)."""
        return lattice_to_ref(self._get(), self.dims, self.comps)

    def to_numpy(self):
        return self.to_torch().contiguous().cpu().numpy().astype(self.np_dtype, copy=False)

    def from_numpy(self, arr):
        if self._put is None:
            raise TypeError(f"field {self.name} is read-only")
        arr = np.asarray(arr)
        want = self.dims + ((self.comps,) if self.comps else ())
        if arr.shape != want:
            raise ValueError(f"from_numpy shape {arr.shape} != field shape {want}")
        self._put(arr)

    def __getitem__(self, idx):
        return self.to_numpy()[idx]

    def __setitem__(self, idx, value):
        a = self.to_numpy().copy()
        a[idx] = value
        self.from_numpy(a)


class ScalarField:
    """A 0-d (``[None]``) or small 1-d diagnostic field."""

    def __init__(self, get, put=None, shape=()):
        self._get = get
        self._put = put
        self.shape = shape

    def __getitem__(self, idx):
        v = self._get()
        if idx is None:
            return v
        return np.asarray(v)[idx]

    def __setitem__(self, idx, value):
        if self._put is None:
            raise TypeError("read-only diagnostic field")
        self._put(idx, value)

    def to_numpy(self):
        return np.asarray(self._get())


class ConstField:
    """Lattice constants (e, e_f, w, S_dig) as read-only fields."""

    def __init__(self, array):
        self._a = np.asarray(array)
        self.shape = self._a.shape[:1] if self._a.ndim else ()

    def to_numpy(self):
        return self._a.copy()

    def __getitem__(self, idx):
        if idx is None:
            return self._a
        return self._a[idx]


class ParticleField:
    """A particle field (n[, comps[, comps]]) backed by a planar device tensor."""

    def __init__(self, tensor_get, shape_tail, np_dtype, put=None, name=""):
        self._get = tensor_get
        self.tail = tuple(shape_tail)
        self.np_dtype = np.dtype(np_dtype)
        self._put = put
        self.name = name

    @property
    def shape(self):
        t = self._get()
        return (t.shape[-1],)

    def to_torch(self):
        t = self._get()
        n = t.shape[-1]
        if not self.tail:
            return t
        return t.reshape(*self.tail, n).permute(len(self.tail), *range(len(self.tail)))

    def to_numpy(self):
        return self.to_torch().contiguous().cpu().numpy().astype(self.np_dtype, copy=False)

    def from_numpy(self, arr):
        t = self._get()
        n = t.shape[-1]
        arr = np.asarray(arr)
        if arr.shape != (n,) + self.tail:
            raise ValueError(f"from_numpy shape {arr.shape} != {(n,) + self.tail}")
        src = torch.as_tensor(np.ascontiguousarray(arr)).to(t.device)
        if self.tail:
            src = src.reshape(n, -1).t()
            t.copy_(src.reshape(t.shape).to(t.dtype))
        else:
            t.copy_(src.to(t.dtype))

    def __getitem__(self, idx):
        return self.to_numpy()[idx]

    def __setitem__(self, idx, value):
        a = self.to_numpy().copy()
        a[idx] = value
        self.from_numpy(a)
