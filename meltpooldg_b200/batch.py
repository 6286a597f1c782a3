"""Batched and served solves on one GPU (mpdg_batch_* / mpdg_serve of include/mpdg.h).

The reference solves one problem per process: LinearSolver::solve
(include/meltpooldg/linear_algebra/linear_solver.hpp:26-134), called from the
heat operation (source/heat/heat_transfer_operation.cpp:300-330) and the
advection-diffusion operation (source/level_set/advection_diffusion_operation.cpp:228-262).
`Batch` keeps many problems' vectors resident on the device and advances all
running problems by one Krylov step per CUDA-graph launch (FP32 operator
apply, FP64 dots, norms, solution and reliable-update defects).  `serve` runs
the library's request loop: Poisson-like arrivals are admitted as memory and
slots free up and leave when they finish.

Problems are unit cubes of nc^3 uniform cells with FE_Q(degree); heat
problems (mass/dt + k0 Laplace) run CG, advection-diffusion problems (vortex
velocity, theta scheme) BiCGStab; both Jacobi-preconditioned.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _capi
from ._capi import OP_ADVDIFF, OP_HEAT, VEL_NONE, VEL_VORTEX, ProblemDesc, SolveReport, check, lib

RUNNING = 1  # report status while a problem runs


@dataclass
class Problem:
    """One batched problem (mpdg_problem_desc)."""
    kind: int = OP_HEAT
    degree: int = 2
    nc: int = 8
    dirichlet: bool = True
    dt: float = 1e-3
    rho_cp: float = 1.0
    k0: float = 1.0
    theta: float = 0.5
    diffusivity: float = 1e-3
    vortex: bool = True
    rel_tolerance: float = 1e-10
    abs_tolerance: float = 0.0
    max_iterations: int = 0
    rhs_seed: int = 0

    def desc(self) -> ProblemDesc:
        d = ProblemDesc()
        d.kind = self.kind
        d.degree = self.degree
        d.nc = self.nc
        d.dirichlet = 1 if self.dirichlet else 0
        d.vel_kind = VEL_VORTEX if (self.kind == OP_ADVDIFF and self.vortex) else VEL_NONE
        d.max_iterations = self.max_iterations
        d.dt = self.dt
        d.rho_cp = self.rho_cp
        d.k0 = self.k0
        d.theta = self.theta
        d.diffusivity = self.diffusivity
        d.rel_tolerance = self.rel_tolerance
        d.abs_tolerance = self.abs_tolerance
        d.rhs_seed = self.rhs_seed
        return d

    @property
    def n_dofs(self) -> int:
        return (self.nc * self.degree + 1) ** 3

    def bytes(self) -> int:
        b, n = C.c_int64(), C.c_int64()
        d = self.desc()
        check(lib().mpdg_problem_bytes(C.byref(d), C.byref(b), C.byref(n)), "mpdg_problem_bytes")
        return int(b.value)

    def rhs(self) -> np.ndarray:
        out = np.empty(self.n_dofs, dtype=np.float64)
        d = self.desc()
        check(lib().mpdg_problem_rhs_host(C.byref(d), out.ctypes.data_as(C.POINTER(C.c_double))),
              "mpdg_problem_rhs_host")
        return out

    def diagonal(self) -> np.ndarray:
        out = np.empty(self.n_dofs, dtype=np.float64)
        d = self.desc()
        check(lib().mpdg_problem_diagonal_host(C.byref(d), out.ctypes.data_as(C.POINTER(C.c_double))),
              "mpdg_problem_diagonal_host")
        return out


class Batch:
    """A set of resident problems advanced together (mpdg_batch)."""

    def __init__(self, budget_bytes: int, capacity: int = 1024, reliable_delta: float = 0.1):
        h = C.c_void_p()
        check(lib().mpdg_batch_create(int(budget_bytes), int(capacity), float(reliable_delta),
                                      C.byref(h)), "mpdg_batch_create")
        self._h = h
        self.capacity = capacity

    def submit(self, problem: Problem, rhs: np.ndarray | None = None) -> int:
        """Admits a problem; raises MpdgError(ERR_BUDGET) when it does not fit."""
        d = problem.desc()
        t = C.c_int64()
        rp = None
        if rhs is not None:
            rhs = np.ascontiguousarray(rhs, dtype=np.float64)
            if rhs.size != problem.n_dofs:
                raise ValueError("rhs has the wrong size")
            rp = rhs.ctypes.data_as(C.POINTER(C.c_double))
        check(lib().mpdg_batch_submit(self._h, C.byref(d), rp, C.byref(t)), "mpdg_batch_submit")
        return int(t.value)

    def try_submit(self, problem: Problem) -> int | None:
        """Admits a problem, or returns None when the budget or the slots are full."""
        try:
            return self.submit(problem)
        except _capi.MpdgError as e:
            if e.status == _capi.ERR_BUDGET:
                return None
            raise

    def run(self, max_steps: int = 1_000_000, poll_steps: int = 8):
        """Runs Krylov steps until no problem runs or max_steps; returns (steps, running)."""
        s, r = C.c_int(), C.c_int()
        check(lib().mpdg_batch_run(self._h, int(max_steps), int(poll_steps), C.byref(s), C.byref(r)),
              "mpdg_batch_run")
        return int(s.value), int(r.value)

    def poll(self, ticket: int) -> dict:
        rep = SolveReport()
        check(lib().mpdg_batch_poll(self._h, int(ticket), C.byref(rep)), "mpdg_batch_poll")
        return rep.as_dict()

    def take(self, ticket: int, n_dofs: int | None = None):
        """(solution or None, report) of a finished problem; releases its slot."""
        rep = SolveReport()
        x = None
        xp = None
        if n_dofs is not None:
            x = np.empty(n_dofs, dtype=np.float64)
            xp = x.ctypes.data_as(C.POINTER(C.c_double))
        check(lib().mpdg_batch_take(self._h, int(ticket), xp, C.byref(rep)), "mpdg_batch_take")
        return x, rep.as_dict()

    def autotune(self):
        """Picks the batched apply's block and tile shape by timing the current
        membership; returns (resident CTAs per SM, its time in ms)."""
        cap, ms = C.c_int(), C.c_double()
        check(lib().mpdg_batch_autotune(self._h, C.byref(cap), C.byref(ms)), "mpdg_batch_autotune")
        return int(cap.value), float(ms.value)

    def shape(self):
        """The batched apply's shape: warps per CTA, tile layout, CTAs per SM."""
        w, t, c = C.c_int(), C.c_int(), C.c_int()
        check(lib().mpdg_batch_shape(self._h, C.byref(w), C.byref(t), C.byref(c)), "mpdg_batch_shape")
        return {"warps_per_cta": w.value, "tile_layout": "conflict-minimal" if t.value else "plain",
                "ctas_per_sm": c.value}

    @property
    def used_bytes(self) -> int:
        b = C.c_int64()
        check(lib().mpdg_batch_used_bytes(self._h, C.byref(b)), "mpdg_batch_used_bytes")
        return int(b.value)

    def serve(self, problems, arrival_s, poll_steps: int = 4, keep_solutions=False):
        """Runs the library's serving loop over requests arriving at arrival_s
        (seconds from the call, ascending).  Returns a dict with per-request
        latency_s, x_norm, reports, the wall time, and the solutions when asked
        (keep_solutions: True for all, or an iterable of request indices)."""
        n = len(problems)
        arr = np.ascontiguousarray(arrival_s, dtype=np.float64)
        if arr.size != n:
            raise ValueError("one arrival time per request")
        descs = (ProblemDesc * max(1, n))(*[p.desc() for p in problems])
        lat = np.zeros(n)
        xn = np.zeros(n)
        reps = (SolveReport * max(1, n))()
        wall = C.c_double()
        sols = None
        xptrs = None
        if keep_solutions is not False and keep_solutions is not None:
            keep = set(range(n)) if keep_solutions is True else set(int(i) for i in keep_solutions)
            sols = [np.empty(p.n_dofs, dtype=np.float64) if i in keep else None
                    for i, p in enumerate(problems)]
            xptrs = (C.POINTER(C.c_double) * max(1, n))(
                *[s.ctypes.data_as(C.POINTER(C.c_double)) if s is not None else C.POINTER(C.c_double)()
                  for s in sols])
        dp = C.POINTER(C.c_double)
        check(lib().mpdg_serve(self._h, descs, arr.ctypes.data_as(dp), n, int(poll_steps), xptrs,
                               lat.ctypes.data_as(dp), xn.ctypes.data_as(dp), reps, C.byref(wall)),
              "mpdg_serve")
        st = (C.c_double * 9)()
        check(lib().mpdg_batch_stats(self._h, st, 9), "mpdg_batch_stats")
        names = ("admit_s", "results_s", "wait_gpu_s", "launch_s", "graph_steps", "admitted", "finished",
                 "max_resident", "polls")
        return {"latency_s": lat, "x_norm": xn, "reports": [reps[i].as_dict() for i in range(n)],
                "wall_s": float(wall.value), "solutions": sols,
                "stats": {k: float(v) for k, v in zip(names, st)}}

    def close(self):
        if getattr(self, "_h", None):
            lib().mpdg_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def solve_batch(problems, budget_bytes: int = 150 * 10**9, poll_steps: int = 8, keep_solutions=True,
                autotune=False):
    """Admits all problems, runs them to completion, returns (solutions, reports)."""
    with Batch(budget_bytes, capacity=max(1, len(problems))) as b:
        tickets = [b.submit(p) for p in problems]
        if autotune:
            b.autotune()
        b.run(poll_steps=poll_steps)
        out, reps = [], []
        for p, t in zip(problems, tickets):
            x, r = b.take(t, p.n_dofs if keep_solutions else None)
            out.append(x)
            reps.append(r)
        return out, reps
