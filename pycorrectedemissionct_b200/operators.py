"""Operator base classes with the reference's interface (``corrct``: ``src/corrct/operators.py``).

``BaseTransform`` mirrors ``operators.py:34-205``: a scipy ``LinearOperator`` whose
``__call__`` applies the direct or the adjoint operator, whose ``.T`` is a shallow copy
with ``is_dir_operator = False`` (``:107-118``) and whose ``absolute()`` returns the
operator itself (``:129-138``).  ``ProjectorOperator`` mirrors ``:283-362`` and routes the
direct / adjoint operator to ``fp`` / ``bp``.  Unchanged corrct solvers only use these
members, so projectors built on them are accepted by corrct's SIRT, MLEM, PDHG and FISTA.
"""

from __future__ import annotations

import copy as cp
from abc import ABC, abstractmethod

import numpy as np
from scipy.sparse.linalg import LinearOperator


class BaseTransform(LinearOperator, ABC):
    """Linear operator with direct/adjoint application (corrct ``operators.py:34-205``)."""

    dir_shape: np.ndarray
    adj_shape: np.ndarray

    def __init__(self) -> None:
        num_cols = int(np.prod(self.dir_shape))
        num_rows = int(np.prod(self.adj_shape))
        super().__init__(np.float32, [num_rows, num_cols])
        self.is_dir_operator = True

    def _matvec(self, x):
        if self.is_dir_operator:
            return self._op_direct(np.reshape(x, self.dir_shape)).flatten()
        return self._op_adjoint(np.reshape(x, self.adj_shape)).flatten()

    def rmatvec(self, x):
        if self.is_dir_operator:
            return self._op_adjoint(np.reshape(x, self.adj_shape)).flatten()
        return self._op_direct(np.reshape(x, self.dir_shape)).flatten()

    def _transpose(self) -> "BaseTransform":
        op_t = cp.copy(self)
        op_t.shape = (self.shape[1], self.shape[0])
        op_t.is_dir_operator = False
        return op_t

    def _adjoint(self) -> "BaseTransform":
        return self._transpose()

    def absolute(self) -> "BaseTransform":
        return self

    def __call__(self, x):
        if self.is_dir_operator:
            return self._op_direct(x)
        return self._op_adjoint(x)

    @abstractmethod
    def _op_direct(self, x): ...

    @abstractmethod
    def _op_adjoint(self, x): ...


class ProjectorOperator(BaseTransform):
    """Projector base: direct = ``fp``, adjoint = ``bp`` (corrct ``operators.py:283-362``)."""

    @property
    def vol_shape(self) -> np.ndarray:
        return self.dir_shape

    @vol_shape.setter
    def vol_shape(self, new_shape) -> None:
        self.dir_shape = np.array(new_shape, ndmin=1, dtype=int)

    @property
    def prj_shape(self) -> np.ndarray:
        return self.adj_shape

    @prj_shape.setter
    def prj_shape(self, new_shape) -> None:
        self.adj_shape = np.array(new_shape, ndmin=1, dtype=int)

    @abstractmethod
    def fp(self, x): ...

    @abstractmethod
    def bp(self, x): ...

    def _op_direct(self, x):
        return self.fp(x)

    def _op_adjoint(self, x):
        return self.bp(x)

    def get_pre_weights(self):
        return None
