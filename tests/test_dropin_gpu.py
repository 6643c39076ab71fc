"""The drop-in Assembler::assemble inside the reference's own solver.

oracle/_ref/libpigfem_ref_b200.so is the reference built from its own sources with its definition
of Assembler::assemble replaced, at link time, by pigfem_b200/drop_in/Assembler_b200.cpp, which
forwards every call to the C ABI (libpigfem_b200.so, sm_100a kernels).  The same RVE is solved
twice by the reference's Problem / SolverNonlinear / SolverNonlinearKSP (adaptive load stepping,
Newton, its direct solver): once with the reference's CPU assembly (oracle/_ref/libpigfem_ref.so)
and once with the drop-in.  The load-step tables must agree: every record's step, repeat,
convergence flag, time and time step, the Newton iteration count of every attempt and the
residual norms (the reference prints 6 significant digits) -- up to the first record where the
reference's own run blows up, after which 1e-16 differences in K decide the path.
"""
import numpy as np
import pytest

from tests.golden.cases import OP, spec_kwargs

pytestmark = pytest.mark.gpu

BL = (50.0, 5e-7, 5e-3, 0.0)   # the bilinear interface of the 512^2 cohesive RVE


@pytest.fixture(scope="module")
def both(oracle_lib):
    if not oracle_lib.available("b200"):
        pytest.skip("drop-in variant of the oracle (oracle/_ref/libpigfem_ref_b200.so) not built")
    return oracle_lib


def _case(law, coh, app):
    return dict(elem_type=0, n=(16, 16), incl=[[0.3, 0.3, 0.12], [0.63, 0.56, 0.13]], coh_law=law, coh=coh,
                subscale=0, seed=1, u_scale=0, isv_scale=0, solve=(1, app))


def _solve(ref, c, variant):
    from pigfem_b200 import newton
    R = ref.RefProblem(ref.ProblemSpec(**spec_kwargs(c)), variant=variant)
    if variant == "b200":
        R.bind_gpu()
    R.set_solver(rel_tol=1e-8, abs_tol=1e-8, max_dt=0.05, min_dt=1e-5, T_final=1.0, max_iter=25)
    steps = newton.parse_reference_log(R.solve())
    state = (R.get("U_final"), R.get("isv_final"))
    R.close()
    return steps, state


def _same_record(a, b, norms=True):
    assert (a.step, a.repeat, a.convergence) == (b.step, b.repeat, b.convergence), (a, b)
    assert a.t == pytest.approx(b.t, rel=1e-5, abs=1e-12) and a.dt == pytest.approx(b.dt, rel=1e-2), (a, b)
    assert len(a.nr_norms) == len(b.nr_norms), (a, b)
    if norms:
        r0 = b.nr_norms[0]
        for x, y in zip(a.nr_norms, b.nr_norms):
            if y > 1e-4 * r0:   # above the linear-solver noise
                assert abs(x - y) <= 2e-5 * y + 1e-12, (x, y)


def test_op_whole_history_and_state(both):
    """Ortiz-Pandolfi interfaces, 0.8 % strain: the whole load-step table and the final state."""
    c = _case(5, OP, 0.008)
    cpu, (U_cpu, isv_cpu) = _solve(both, c, "cpu")
    gpu, (U_gpu, isv_gpu) = _solve(both, c, "b200")
    assert len(cpu) == len(gpu) and len(cpu) >= 20
    for a, b in zip(gpu, cpu):
        _same_record(a, b)
    assert np.linalg.norm(U_gpu - U_cpu) <= 1e-9 * np.linalg.norm(U_cpu)
    assert np.abs(isv_gpu - isv_cpu).max() <= 1e-9 * np.abs(isv_cpu).max()


def test_bilinear_tension_until_the_reference_breaks_down(both):
    """The bilinear law of the 512^2 cohesive RVE (sigma_c 50, delta_c1 5e-7, delta_c2 5e-3) under
    2 % strain on the 16^2 two-fiber RVE.  The reference's own run converges step by step until a
    Newton attempt blows up (its residual grows from about 22 to about 6e8 near t = 0.35) and,
    after further cut-backs, stops on a zero or non-finite pivot of its direct solver before the
    end of the ramp.  The drop-in run must reproduce every converged record before that first
    failed attempt to the printed digits, and it must not finish the ramp either (in the blown-up
    attempt 1e-16 differences in K decide how far the run gets)."""
    c = _case(1, BL, 0.02)
    cpu, _ = _solve(both, c, "cpu")
    gpu, _ = _solve(both, c, "b200")
    first_fail = next(i for i, s in enumerate(cpu) if s.convergence != 1)
    assert cpu[first_fail].t < 0.5 and max(cpu[first_fail].nr_norms) > 1e4 * cpu[first_fail].nr_norms[0]
    assert len(gpu) >= first_fail
    for a, b in zip(gpu[:first_fail], cpu[:first_fail]):
        _same_record(a, b)
    # neither run reaches the end of the load ramp with this law
    assert cpu[-1].t < 1.0 - 1e-9 and gpu[-1].t < 1.0 - 1e-9
