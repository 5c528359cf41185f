"""Field adapter: a torch tensor with the slice of the Taichi field API the
reference's callers and tests use (``shape``, ``dtype``, ``to_numpy``,
``from_numpy``, ``fill``, element get/set with ``[i, j, k]`` / ``[None]``).

Scalar fields have shape ``shape``; vector fields add a trailing axis of size
``n``; matrix fields add ``(n, m)``.  Element reads return Python numbers for
scalar fields and tuples for vector / matrix fields (rows for matrices).
"""

from __future__ import annotations

import numpy as np
import torch


class Field:
    def __init__(self, shape, dtype: torch.dtype, *, n: int | None = None, m: int | None = None, device=None, tensor=None):
        self.shape = tuple(int(s) for s in (shape if isinstance(shape, (tuple, list)) else (shape,)))
        self.n = n
        self.m = m
        self.dtype = dtype
        trailing = () if n is None else ((n,) if m is None else (n, m))
        if tensor is None:
            tensor = torch.zeros(self.shape + trailing, dtype=dtype, device=device)
        self.tensor = tensor

    # -- pointers for the C ABI --
    def ptr(self) -> int:
        if not self.tensor.is_contiguous():
            raise RuntimeError("field storage must be contiguous")
        return self.tensor.data_ptr()

    def numel_cells(self) -> int:
        return int(np.prod(self.shape)) if self.shape else 1

    # -- bulk transfer --
    def to_numpy(self) -> np.ndarray:
        return self.tensor.detach().cpu().numpy().copy()

    def to_torch(self, device=None) -> torch.Tensor:
        return self.tensor.clone() if device is None else self.tensor.to(device).clone()

    def from_numpy(self, array) -> None:
        src = torch.as_tensor(np.ascontiguousarray(array))
        if tuple(src.shape) != tuple(self.tensor.shape):
            raise ValueError(f"from_numpy shape {tuple(src.shape)} does not match field shape {tuple(self.tensor.shape)}")
        self.tensor.copy_(src.to(self.dtype))

    def from_torch(self, tensor: torch.Tensor) -> None:
        if tuple(tensor.shape) != tuple(self.tensor.shape):
            raise ValueError("from_torch shape mismatch")
        self.tensor.copy_(tensor.to(self.dtype))

    def copy_from(self, other: "Field") -> None:
        self.tensor.copy_(other.tensor)

    def fill(self, value) -> None:
        self.tensor.fill_(value)

    # -- element access --
    def _key(self, index):
        if index is None:
            if self.shape:
                raise IndexError("None index is only valid for 0-D fields")
            return ()
        if not isinstance(index, tuple):
            index = (index,)
        if len(index) != len(self.shape):
            raise IndexError(f"field of rank {len(self.shape)} indexed with {len(index)} indices")
        return tuple(int(i) for i in index)

    def __getitem__(self, index):
        value = self.tensor[self._key(index)].detach().cpu()
        if self.n is None:
            return value.item()
        if self.m is None:
            return tuple(v.item() for v in value)
        return tuple(tuple(v.item() for v in row) for row in value)

    def __setitem__(self, index, value) -> None:
        key = self._key(index)
        if self.n is None:
            self.tensor[key] = value
        else:
            self.tensor[key] = torch.as_tensor(np.asarray(value), dtype=self.dtype)

    def __repr__(self) -> str:
        return f"Field(shape={self.shape}, n={self.n}, m={self.m}, dtype={self.dtype})"
