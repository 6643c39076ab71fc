"""Load stepping with Newton-Raphson on the device: the reference's nonlinear solver loop driven
through the C ABI.

Restates SolverNonlinear::solve (src/SolverNonlinear.cpp:70-328, adaptive load stepping),
SolverNonlinear::update_time_step (src/SolverNonlinear.cpp:386-422) and
SolverNonlinearKSP::nonlinearStep (src/SolverNonlinearKSP.cpp:55-157, the Newton loop) with the
same control flow, tolerances and logging quantities.  Every assembly runs on the device
(pg_assemble_device) and the residual norm is the device's fixed-order FP64 reduction
(pg_residual_norm); the displacement, the CSR values and the internal variables stay resident in
HBM.  The Newton correction is solved by the device Jacobi-PCG (positive definite tangents) or by
a host sparse direct factorisation, the counterpart of the reference's MUMPS Cholesky, which also
takes the indefinite tangents that softening interfaces produce.

The reference's last-resort explicit solver (entered after 20 repeats of one load step or a time
step below min_dt) is not restated: the driver stops with NewtonFailure there instead.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field
from typing import List

import numpy as np

from . import capi


class NewtonFailure(RuntimeError):
    pass


@dataclass
class StepRecord:
    """One line of the reference's load-step table (LStp, T, TStep, Rpt, Cnv, Res)."""
    step: int
    t: float
    dt: float
    repeat: int
    convergence: int
    res_norm: float
    nr_norms: List[float] = field(default_factory=list)
    nr_times: List[float] = field(default_factory=list)   # seconds of each Newton correction


@dataclass
class SolveResult:
    steps: List[StepRecord]
    U_free: np.ndarray
    isv: np.ndarray
    failed: str = ""      # why the run stopped early (raise_on_failure=False), else empty

    def log(self) -> str:
        """The run's solver log in the reference's text (format_log)."""
        return format_log(self.steps)


class LoadStepper:
    """The reference's load-stepping and Newton control flow over four operations a subclass
    provides: set the load (prescribed values at t/T_final), assemble and return the residual
    norm, solve for and apply the Newton correction, and save / restore / commit the state."""

    MAX_TIME_STEP_REPEAT = 20
    DECREASE, INCREASE = 0.25, 1.5

    def __init__(self, T_final: float = 1.0, max_dt: float = 0.05, min_dt: float = 1e-5, rel_tol: float = 1e-8,
                 abs_tol: float = 1e-8, max_iter: int = 25):
        self.T_final, self.max_dt, self.min_dt = T_final, max_dt, min_dt
        self.rel_tol, self.abs_tol, self.max_iter = rel_tol, abs_tol, max_iter

    # operations
    def set_load(self, t_frac: float): raise NotImplementedError
    def assemble(self, t_frac: float) -> float: raise NotImplementedError
    def correct(self) -> bool: raise NotImplementedError
    def save(self): raise NotImplementedError
    def restore(self): raise NotImplementedError
    def commit(self): raise NotImplementedError
    def result(self, records) -> "SolveResult": raise NotImplementedError

    def nonlinear_step(self, t_frac: float):
        """SolverNonlinearKSP::nonlinearStep: returns (converged, final norm, norms)."""
        res = self.assemble(t_frac)
        res0 = res
        norms = [res]
        self._times = times = []
        it = 0
        increase = 0
        while True:
            t0 = time.perf_counter()
            ok = self.correct()
            times.append(time.perf_counter() - t0)
            if not ok:
                return False, float("nan"), norms
            prev = res
            res = self.assemble(t_frac)
            norms.append(res)
            it += 1
            if res < self.rel_tol * res0 or res < self.abs_tol:
                return True, res, norms
            if not math.isfinite(res):
                return False, res, norms
            if it >= self.max_iter:
                return False, res, norms
            increase = increase + 1 if res > prev else 0
            if increase >= 3:
                return False, res, norms

    def solve(self, raise_on_failure: bool = True) -> "SolveResult":
        """SolverNonlinear::solve.  With raise_on_failure=False a run the reference would hand to
        its explicit solver returns the records so far with `failed` set."""
        try:
            return self._solve()
        except NewtonFailure as e:
            if raise_on_failure:
                raise
            res = self.result(self._records)
            res.failed = str(e)
            return res

    def _solve(self) -> "SolveResult":
        dt = self.max_dt
        t = 0.0
        step_iter = 0
        records: List[StepRecord] = []
        self._records = records
        self.save()
        while t < self.T_final:
            repeat = 0
            converged = False
            while not converged:
                if repeat == self.MAX_TIME_STEP_REPEAT or dt < self.min_dt:
                    raise NewtonFailure(f"load step {step_iter + 1} at t = {t}: the reference would enter its "
                                        "explicit solver here")
                repeat += 1
                t_frac = (t + dt) / self.T_final
                self.set_load(t_frac)
                converged, res, norms = self.nonlinear_step(t_frac)
                if converged:
                    conv = 1
                    t += dt
                else:
                    conv = -1
                    self.restore()
                records.append(StepRecord(step_iter + 1, t, dt, repeat, conv, res, norms, list(self._times)))
                dt, t = self._update_time_step(dt, t, converged, repeat)
            self.commit()
            self.save()
            step_iter += 1
        return self.result(records)

    def _update_time_step(self, dt: float, t: float, converged: bool, repeat: int):
        """SolverNonlinear::update_time_step (no rate limits, no problem-controlled steps)."""
        if not converged:
            dt = self.DECREASE * dt
        elif repeat == 1:
            dt = self.INCREASE * dt
        remaining = self.T_final - t
        if dt > self.max_dt:
            dt = self.max_dt
        if dt > remaining:
            if remaining >= self.min_dt:
                dt = remaining
            else:
                t = self.T_final
        return dt, t


class NewtonSolver(LoadStepper):
    """Drives one context (`capi.Problem`) through the load ramp t/T_final of its prescribed
    displacements (Dirichlet mode) or macroscale strain (subscale mode).  Assembly, residual norm,
    state and internal variables live on the device.  The Newton correction K_ff dU = -P_f is
    solved by the device Jacobi-PCG (linear_solver="pcg"; K_ff must stay positive definite) or,
    like the reference's direct Cholesky, by a direct sparse factorisation on the host
    (linear_solver="direct": K_ff values copied back once per Newton iteration), which also
    handles the indefinite tangents of softening interfaces."""

    def __init__(self, problem: capi.Problem, T_final: float = 1.0, max_dt: float = 0.05, min_dt: float = 1e-5,
                 rel_tol: float = 1e-8, abs_tol: float = 1e-8, max_iter: int = 25, fp32: bool = False,
                 linear_solver: str = "direct", pcg_rtol: float = 1e-13, pcg_max_it: int = 200000):
        super().__init__(T_final, max_dt, min_dt, rel_tol, abs_tol, max_iter)
        import torch
        self.torch = torch
        self.P = problem
        self.flags = capi.FUNC | capi.JAC | (capi.FP32 if fp32 else 0)
        if linear_solver not in ("pcg", "direct"):
            raise ValueError(linear_solver)
        self.linear_solver = linear_solver
        self.pcg_rtol, self.pcg_max_it = pcg_rtol, pcg_max_it
        _, dofs, dirichlet = problem.nodes()
        dev = torch.device("cuda")
        self.node_dofs = torch.from_numpy(dofs.reshape(-1).astype(np.int64)).to(dev)
        self.dirichlet = torch.from_numpy(np.ascontiguousarray(dirichlet, dtype=np.float64)).to(dev)
        nf, nc = problem.n_free, problem.n_const
        self.nf, self.nc = nf, nc
        self.U = torch.zeros(nf + nc, dtype=torch.float64, device=dev)      # free then constrained
        self.U_node = torch.zeros(problem.n_nodes * problem.dim, dtype=torch.float64, device=dev)
        self.dx = torch.zeros(max(nf, 1), dtype=torch.float64, device=dev)
        self.stream = torch.cuda.current_stream()
        problem.set_stream(self.stream.cuda_stream)
        self.pcg_iterations = 0
        if linear_solver == "direct":
            rp, ci, _ = problem.pattern(0)
            self._rp, self._ci = rp, ci
            self._kff_host = torch.empty(max(len(ci), 1), dtype=torch.float64).pin_memory()
            self._pf_host = torch.empty(max(nf, 1), dtype=torch.float64).pin_memory()

    def set_load(self, t_frac: float):
        if self.nc:
            self.U[self.nf:] = self.dirichlet * t_frac

    def assemble(self, t_frac: float) -> float:
        """Assembler::assemble with the current U; returns ||F_ext,f - P_int,f|| (F_ext,f = 0)."""
        self.U_node.copy_(self.U[self.node_dofs])
        self.P.assemble_device(self.U_node.data_ptr(), t_frac, self.flags)
        return self.P.residual_norm()

    def correct(self) -> bool:
        """K_ff dU = F_ext,f - P_int,f = -P_f."""
        torch = self.torch
        K, pf, _ = self.P.device_outputs()
        if self.linear_solver == "pcg":
            self.dx.zero_()
            try:
                it, _ = self.P.pcg_solve(pf, self.dx.data_ptr(), 1, self.pcg_rtol, self.pcg_max_it)
            except capi.PigfemError:
                return False
            self.pcg_iterations += int(it[0])
            self.U[: self.nf] -= self.dx[: self.nf]
            return True
        import scipy.sparse as sp
        import scipy.sparse.linalg as spla
        nnz = len(self._ci)
        self._kff_host[:nnz].copy_(capi.device_view(K[0], nnz), non_blocking=True)
        self._pf_host[: self.nf].copy_(capi.device_view(pf, self.nf), non_blocking=True)
        self.stream.synchronize()
        A = sp.csr_matrix((self._kff_host.numpy()[:nnz], self._ci, self._rp), shape=(self.nf, self.nf)).tocsc()
        rhs = -self._pf_host.numpy()[: self.nf]
        try:
            du = spla.spsolve(A, rhs)
        except RuntimeError:
            return False
        if not np.all(np.isfinite(du)):
            return False
        self.U[: self.nf] += torch.from_numpy(du).to(self.U.device)
        return True

    def save(self):
        self._prev_Uf = self.U[: self.nf].clone()

    def restore(self):
        self.U[: self.nf] = self._prev_Uf

    def commit(self):
        self.P.commit_isv()

    def result(self, records):
        self.torch.cuda.synchronize()
        isv = self.P.get_isv(trial=False) if self.P.n_isv else np.zeros(0)
        return SolveResult(records, self.U[: self.nf].cpu().numpy(), isv)


LOG_HEADER = ("\n\nStarting time step algorithm.\n"
              "Cnv cheatsheet:\n  1: Converged\n -1: NR-diverged\n -2: Large damage rate\n"
              "LStp      T(s)      TStep(s)    Rpt   Cnv    Res\n"
              "----   ----------   --------    ---   ---  --------\n")


def _g(x: float) -> str:
    """A double as a C++ stream prints it by default (%g, 6 significant digits)."""
    return "%g" % x


def format_log(records: List[StepRecord]) -> str:
    """The solver log of a run in the reference's own text: the table header
    (src/SolverNonlinear.cpp:111-114), the Newton lines of every attempt
    (src/SolverNonlinearKSP.cpp:89, 117), "REPEATING LOADSTEP" after an attempt that failed
    (src/SolverNonlinear.cpp:225) and the load-step line (src/SolverNonlinear.cpp:241-246), so that
    a run's log reads, and parses, like a reference run's."""
    out = [LOG_HEADER]
    for r in records:
        for k, res in enumerate(r.nr_norms):
            if k == 0:
                out.append("\tNR iteration: 0 Residual: %s\n" % _g(res))
            else:
                dt = r.nr_times[k - 1] if k - 1 < len(r.nr_times) else 0.0
                out.append("\tNR iteration: %d Iteration_Time: %s \tResidual: %s\n" % (k, _g(dt), _g(res)))
        if r.convergence != 1:
            out.append("REPEATING LOADSTEP\n")
        out.append(" %d     %1.5e  %1.2e     %d     %d   %1.2e\n" % (r.step, r.t, r.dt, r.repeat, r.convergence,
                                                                      r.res_norm))
    return "".join(out)


def parse_reference_log(log: str):
    """Load-step table and Newton norms from the reference's solver log (the lines printed by
    src/SolverNonlinear.cpp:241-246 and src/SolverNonlinearKSP.cpp:71, 106)."""
    steps, nr, times = [], [], []
    for line in log.splitlines():
        s = line.strip()
        if s.startswith("NR iteration:"):
            nr.append(float(s.split("Residual:")[-1]))
            if "Iteration_Time:" in s:
                times.append(float(s.split("Iteration_Time:")[1].split()[0]))
            continue
        parts = s.split()
        if len(parts) == 6 and parts[0].isdigit():
            try:
                steps.append(StepRecord(int(parts[0]), float(parts[1]), float(parts[2]), int(parts[3]), int(parts[4]),
                                        float(parts[5]), nr, times))
            except ValueError:
                continue
            nr, times = [], []
    return steps
