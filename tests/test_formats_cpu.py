"""The reference's output formats, on CPU against the reference's own writers (run live):

* the homogenization CSV (WriterHomogenization) written here equals, character for character,
  the file the reference writes for the same macroscale strain and homogenized stress, at step 0
  (new file) and step 1 (appended), and without a homogenized value;
* the solver log (the load-step table of SolverNonlinear::solve and the Newton lines of
  SolverNonlinearKSP::nonlinearStep) formatted here from a run's records equals the reference's
  log text, repeated load steps included.
"""
import os

import numpy as np
import pytest

from tests.golden.cases import CASES, OP, spec_kwargs


def _ref(oracle, c):
    return oracle.RefProblem(oracle.ProblemSpec(**spec_kwargs(c)))


@pytest.mark.parametrize("name", ["lin_tri3_subscale", "lin_tet4_subscale"])
def test_homogenization_csv_matches_reference_writer(oracle_lib, name, tmp_path):
    from pigfem_b200 import writers
    R = _ref(oracle_lib, CASES[name])
    nv = 6 if CASES[name]["elem_type"] == 2 else 3
    e = np.array([1.0, -0.25, 0.5, 0.125, -0.75, 0.3][:nv])
    R.set_macro(e)
    ref_file, our_file = str(tmp_path / "ref.csv"), str(tmp_path / "ours.csv")
    U = np.zeros(R.n_free + R.n_const)
    for step, t in enumerate((0.3, 1.0)):
        R.assemble(U, None, t)
        h = R.homogenize()
        R.write_homogenization(ref_file, t, step)
        writers.write_homogenization(our_file, t, step, e * t, h)
    ref_txt, our_txt = open(ref_file).read(), open(our_file).read()
    assert our_txt == ref_txt
    assert len(our_txt.splitlines()) == 2 and len(our_txt.splitlines()[0].split(",")) == 1 + 2 * nv
    R.close()


def test_homogenization_csv_without_homogenized_value(oracle_lib, tmp_path):
    from pigfem_b200 import writers
    R = _ref(oracle_lib, CASES["lin_tri3_subscale"])
    e = np.array([0.1, 0.2, 1.0 / 3.0])
    R.set_macro(e)
    R.assemble(np.zeros(R.n_free + R.n_const), None, 0.7)
    R.write_homogenization(str(tmp_path / "ref.csv"), 0.7, 0)
    assert open(tmp_path / "ref.csv").read() == writers.homogenization_row(0.7, e * 0.7)
    R.close()


@pytest.mark.parametrize("law,app", [(5, 0.02), (6, 0.02)], ids=["op", "opnu_cutbacks"])
def test_solver_log_matches_reference_text(oracle_lib, law, app):
    """format_log over the records of a reference run gives back the reference's log text; the
    OPNU run repeats three load steps, so its log holds "REPEATING LOADSTEP" lines."""
    from pigfem_b200 import newton
    c = dict(elem_type=0, n=(16, 16), incl=[[0.3, 0.3, 0.12], [0.63, 0.56, 0.13]], coh_law=law, coh=OP, subscale=0,
             seed=1, u_scale=0, isv_scale=0, solve=(1, app))
    R = _ref(oracle_lib, c)
    R.set_solver(rel_tol=1e-8, abs_tol=1e-8, max_dt=0.05, min_dt=1e-5, T_final=1.0, max_iter=25)
    log = R.solve()
    R.close()
    recs = newton.parse_reference_log(log)
    assert recs and all(len(r.nr_times) == len(r.nr_norms) - 1 for r in recs)
    assert newton.format_log(recs) == log
    if law == 6:
        assert "REPEATING LOADSTEP" in log


def test_solver_log_round_trip_of_own_records():
    """Records of a run here (full-precision norms and times) print in the reference's layout and
    parse back to the printed precision."""
    from pigfem_b200 import newton
    recs = [newton.StepRecord(1, 0.05, 0.05, 1, 1, 3.2e-10, [22.3212345, 0.0596252001, 3.2e-10], [1.1e-3, 1.2e-3]),
            newton.StepRecord(2, 0.05, 0.05, 1, -1, float("nan"), [21.0, 40.0], [1e-3]),
            newton.StepRecord(2, 0.0625, 0.0125, 2, 1, 1e-9, [5.0, 1e-9], [2e-3])]
    txt = newton.format_log(recs)
    assert txt.startswith(newton.LOG_HEADER)
    assert txt.count("REPEATING LOADSTEP") == 1
    back = newton.parse_reference_log(txt)
    assert [(r.step, r.repeat, r.convergence) for r in back] == [(r.step, r.repeat, r.convergence) for r in recs]
    for a, b in zip(back, recs):
        assert np.allclose(a.nr_norms, b.nr_norms, rtol=1e-5)
        assert abs(a.t - b.t) <= 1e-5 * b.t
    assert " 1     5.00000e-02  5.00e-02     1     1   3.20e-10" in txt.splitlines()


def test_served_homogenization_as_reference_csv():
    """A served homogenization result (the modulus C, column k = <sigma> under e_k) as the
    reference's CSV rows: t = 1, the unit strain, then the column."""
    from pigfem_b200 import serving, writers
    C = np.array([[10.0, 2.5, 0.0], [2.5, 10.0, 0.0], [0.0, 0.0, 3.75]]) * 1e3 + 1.0 / 3.0
    txt = serving.homogenization_csv(serving.Result(0, "homogenize", 8, {"C": C}))
    rows = txt.splitlines()
    assert len(rows) == 3
    for k, row in enumerate(rows):
        e = np.zeros(3)
        e[k] = 1.0
        assert row + "\n" == writers.homogenization_row(1.0, e, C[:, k])
        vals = [float(v) for v in row.split(",")]
        assert vals[0] == 1.0 and vals[1:4] == list(e)
        assert np.allclose(vals[4:], C[:, k], rtol=1e-15, atol=0)   # 16 significant digits
