"""Device matrix and vector (the GenericMatrix/GenericVector surface the
assembler writes into; dolfin/la/EigenMatrix.h, EigenVector.h).

Matrix values live in a torch float64 CUDA tensor laid out as the pattern's
sorted CSR (int32 rowptr/cols, as Eigen::SparseMatrix<double, RowMajor, int>);
``data()`` returns host copies like EigenMatrix.data() in the reference's
Python layer (python/src/la.cpp:768-790).
"""
from __future__ import annotations

import numpy as np


class Matrix:
    def __init__(self, pattern=None):
        self._pattern = pattern
        self._vals = None
        if pattern is not None:
            self._alloc()

    def _alloc(self):
        import torch
        self._vals = torch.zeros(self._pattern.nnz(), dtype=torch.float64, device="cuda")

    # GenericTensor::empty (dolfin/la/GenericTensor.h)
    def empty(self):
        return self._pattern is None

    def init(self, pattern):
        self._pattern = pattern
        self._alloc()

    @property
    def pattern(self):
        return self._pattern

    def values_tensor(self):
        """The device value array (torch float64, length nnz)."""
        return self._vals

    def zero(self):
        self._vals.zero_()

    def apply(self, mode="add"):
        pass  # values are final when the kernel completes (EigenMatrix::apply is makeCompressed)

    def size(self, dim):
        return self._pattern.nrows

    def nnz(self):
        return self._pattern.nnz()

    def data(self, deepcopy=True):
        rp, cols = self._pattern.csr_host()
        return rp, cols, self._vals.detach().cpu().numpy()

    def data_device(self):
        rp, cols = self._pattern.csr_device()
        return rp, cols, self._vals

    def norm(self, norm_type="frobenius"):
        if norm_type != "frobenius":
            raise ValueError("matrix norms: 'frobenius' only")
        return float(self._vals.norm().item())

    def sparray(self):
        import scipy.sparse as sp
        rp, cols, vals = self.data()
        n = self._pattern.nrows
        return sp.csr_matrix((vals, cols, rp), shape=(n, n))

    def array(self):
        return self.sparray().toarray()

    def mult(self, x, y):
        """y = A x with the assembled CSR (for checking the matrix-free action)."""
        import torch
        rp, cols, vals = self.data_device()
        A = torch.sparse_csr_tensor(rp.long(), cols.long(), vals, size=(self.size(0), self.size(0)))
        y.tensor().copy_(A @ x.tensor())


class Vector:
    def __init__(self, x=None, n=None):
        import torch
        if x is None:
            x = torch.zeros(int(n or 0), dtype=torch.float64, device="cuda")
        self._x = x

    def tensor(self):
        return self._x

    def empty(self):
        return self._x.numel() == 0

    def size(self):
        return int(self._x.numel())

    def zero(self):
        self._x.zero_()

    def apply(self, mode="add"):
        pass

    def get_local(self):
        return self._x.detach().cpu().numpy()

    def norm(self, norm_type="l2"):
        if norm_type == "l2":
            return float(self._x.norm().item())
        if norm_type == "l1":
            return float(self._x.abs().sum().item())
        if norm_type == "linf":
            return float(self._x.abs().max().item())
        raise ValueError(norm_type)

    def sum(self):
        return float(self._x.sum().item())
