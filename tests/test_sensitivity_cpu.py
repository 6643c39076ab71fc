"""The reference's material sensitivity pass (the oracle, no GPU), pinned by two properties of
linear elasticity on meshes of one material (no fibers), where the pass is plain calculus:

* D is proportional to E, so E dP/dE equals the internal force P_int(U) itself;
* dP/dnu equals the central difference (P(nu + h) - P(nu - h)) / 2h of the reference's own
  assembly to O(h^2).
"""
import numpy as np
import pytest

from tests.golden.cases import spec_kwargs


def _spec(ref, elem_type, n, nu=0.35, sens_param=0, subscale=False):
    c = dict(elem_type=elem_type, n=n, incl=np.zeros((0, 3 if elem_type != 2 else 4)), coh_law=0, coh=(0, 0, 0, 0),
             subscale=int(subscale), eps_macro=(0.0,) * (3 if elem_type != 2 else 6))
    kw = spec_kwargs(c)
    kw["nu_matrix"] = nu
    return ref.ProblemSpec(**kw, sens_mat=1, sens_param=sens_param)


@pytest.mark.parametrize("elem_type,n", [(0, (6, 5)), (1, (5, 4)), (2, (3, 3, 2))])
def test_E_sensitivity_is_the_internal_force_over_E(oracle_lib, elem_type, n):
    ref = oracle_lib
    spec = _spec(ref, elem_type, n)
    R = ref.RefProblem(spec)
    U = np.random.default_rng(7).uniform(-1e-3, 1e-3, R.n_free + R.n_const)
    dPf, dPp = R.sensitivity(U)
    R.assemble(U, None, 1.0, func=True, jac=False)
    Pf, Pp = R.get("P_f"), R.get("P_p")
    E = spec.E_matrix
    assert np.abs(E * dPf - Pf).max() <= 1e-13 * np.abs(Pf).max()
    assert np.abs(E * dPp - Pp).max() <= 1e-13 * np.abs(Pp).max()
    R.close()


@pytest.mark.parametrize("elem_type,n", [(0, (6, 5)), (2, (3, 3, 2))])
def test_nu_sensitivity_matches_a_central_difference(oracle_lib, elem_type, n):
    ref = oracle_lib
    nu, h = 0.35, 1e-5
    R = ref.RefProblem(_spec(ref, elem_type, n, nu=nu, sens_param=4))
    U = np.random.default_rng(8).uniform(-1e-3, 1e-3, R.n_free + R.n_const)
    dPf, _ = R.sensitivity(U)
    P = []
    for v in (nu + h, nu - h):
        Rv = ref.RefProblem(_spec(ref, elem_type, n, nu=v))
        Rv.assemble(U, None, 1.0, func=True, jac=False)
        P.append(Rv.get("P_f"))
        Rv.close()
    fd = (P[0] - P[1]) / (2 * h)
    assert np.abs(dPf - fd).max() <= 1e-7 * np.abs(fd).max()
    R.close()
