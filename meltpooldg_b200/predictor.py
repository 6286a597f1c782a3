"""Least-squares-projection predictor (LeastSquaresProjection,
include/meltpooldg/linear_algebra/predictor.hpp:19-86) on the device.

    lsp = LeastSquaresProjection(history)      # old solutions, newest first
    n_used = lsp.vmult(op, solution, rhs)      # solution = sum_s c_s history[s]

The images A history[s] come from one multi-vector apply; the modified
Gram-Schmidt recurrence, its stopping rule and the back substitution are the
reference's (mpdg_predict_lsq)."""
from __future__ import annotations

import ctypes as C

from . import _capi as A


class LeastSquaresProjection:
    def __init__(self, solution_history, n_old_solutions=None):
        n = len(solution_history) if n_old_solutions is None else int(n_old_solutions)
        if n > len(solution_history):
            raise ValueError("more old solutions requested than the history holds")
        self.old_solution = list(solution_history[:n])
        self.n_used = 0

    def vmult(self, op, solution, rhs):
        """Writes the prediction into `solution`; returns how many old solutions
        entered it (fewer than given when their images became dependent)."""
        n = len(self.old_solution)
        olds = (C.c_void_p * n)(*[t.data_ptr() for t in self.old_solution])
        used = C.c_int(0)
        A.check(A.lib().mpdg_predict_lsq(op._h, n, olds, C.c_void_p(rhs.data_ptr()),
                                         C.c_void_p(solution.data_ptr()), C.byref(used)), "predict_lsq")
        self.n_used = int(used.value)
        return self.n_used
