"""Function and Constant (dolfin/function/Function.h, Constant.h).

A Function owns its dof vector on the GPU (a torch float64 tensor); the
engine reads it directly (Function::restrict's gather happens inside the
assembly kernels).
"""
from __future__ import annotations

import numpy as np

from .ufl import _NPROBE, Expr


class Constant(Expr):
    def __init__(self, value, cell=None, name=None):
        v = np.atleast_1d(np.asarray(value, np.float64))
        if v.ndim != 1 or v.size > 3:
            raise ValueError("Constant: scalar or vector of size <= 3")
        self._v = v
        self.ops = ()
        self.shape = () if v.size == 1 and np.ndim(value) == 0 else (v.size,)

    def values(self):
        return self._v.copy()

    def value_size(self):
        return self._v.size

    def __float__(self):
        if self._v.size != 1:
            raise TypeError("vector Constant")
        return float(self._v[0])

    def ev(self, env):
        if not self.shape:
            return np.full((_NPROBE,), self._v[0])
        return np.broadcast_to(self._v, (_NPROBE, self._v.size)).copy()


class Function(Expr):
    """P1 (or P2) Lagrange function with a device dof vector."""

    def __init__(self, V, values=None, name=None):
        import torch
        self._V = V
        self.ops = ()
        vs = V.value_size()
        self.shape = () if vs == 1 else (vs,)
        if values is None:
            self._x = torch.zeros(V.dim(), dtype=torch.float64, device="cuda") \
                if torch.cuda.is_available() else torch.zeros(V.dim(), dtype=torch.float64)
        else:
            t = torch.as_tensor(values, dtype=torch.float64)
            if t.numel() != V.dim():
                raise ValueError("Function values have the wrong size")
            self._x = t.to("cuda") if torch.cuda.is_available() else t.clone()
        self.name = name or "f"

    def function_space(self):
        return self._V

    def vector(self):
        from .la import Vector
        return Vector(self._x)

    def tensor(self):
        """The device dof vector (torch float64)."""
        return self._x

    def vertex_tensor(self):
        """Values by vertex index of a P1 function (the engine's coefficient
        layout): the dof vector itself, or gathered for a reordered space.
        The gathered copy is kept on the object so that it outlives the
        asynchronous kernels that read it."""
        V = self._V
        if not V.reordered():
            return self._x
        import torch
        idx = torch.as_tensor(V.node_numbers().astype("int64"), device=self._x.device)
        self._vtx = self._x[idx]
        return self._vtx

    def assign_values(self, values):
        import torch
        self._x.copy_(torch.as_tensor(values, dtype=torch.float64))

    def ev(self, env):
        return env["f"][self]

    def __hash__(self):
        return id(self)

    def __eq__(self, other):
        return self is other
