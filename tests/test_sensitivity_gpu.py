"""Material sensitivity of the internal force through the C ABI (pg_material_sensitivity) against
the reference's own SensitivityParameter::assemble_dPdd run live: every parameter of the linear
elastic matrix and fiber materials, on tri3 / quad4 / tet4 meshes with cut elements (polygon
sub-elements, where the reference reads the gradients of the element's leading points), periodic
meshes and bounding plies.  Bar: 1e-12 relative (FP64, the same sums up to rounding)."""
import numpy as np
import pytest

from tests.golden.cases import CASES, spec_kwargs

pytestmark = pytest.mark.gpu

TOL = 1e-12


def rel(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


CASES_PARAMS = [(name, mat, p) for name in ("lin_tri3_one_fiber", "lin_tri3_polygon", "lin_tet4_one_sphere")
                for mat in (0, 1) for p in range(5)]
CASES_PARAMS += [(name, mat, p) for name in ("lin_quad4_one_fiber", "lin_tri3_subscale", "lin_tet4_subscale",
                                             "lin_tri3_ply_cut", "lin_quad4_two_fibers_one_element")
                 for mat in (0, 1) for p in (0, 4)]


@pytest.mark.parametrize("name,mat,param", CASES_PARAMS)
def test_material_sensitivity_matches_reference(oracle_lib, name, mat, param):
    import torch
    from pigfem_b200 import capi
    ref = oracle_lib
    kw = spec_kwargs(CASES[name])
    R = ref.RefProblem(ref.ProblemSpec(**kw, sens_mat=mat + 1, sens_param=param))
    P = capi.Problem(capi.ProblemDesc(**kw))
    _, dofs, _ = P.nodes()
    U = np.random.default_rng(100 + param).uniform(-1e-3, 1e-3, R.n_free + R.n_const)
    ref_f, ref_p = R.sensitivity(U)
    dU = torch.from_numpy(np.ascontiguousarray(U[dofs.reshape(-1)])).cuda()
    f = torch.full((P.n_free,), float("nan"), dtype=torch.float64, device="cuda")
    p = torch.full((max(1, P.n_const),), float("nan"), dtype=torch.float64, device="cuda")
    P.material_sensitivity(dU.data_ptr(), mat, param, f.data_ptr(), p.data_ptr() if P.n_const else 0)
    got_f = f.cpu().numpy()
    assert np.isfinite(got_f).all()
    assert rel(got_f, ref_f) <= TOL, rel(got_f, ref_f)
    if P.n_const:
        got_p = p.cpu().numpy()
        assert np.isfinite(got_p).all()
        assert rel(got_p, ref_p) <= TOL, rel(got_p, ref_p)
    R.close()
    P.close()


def test_material_sensitivity_refuses_cohesive_problems():
    import torch
    from pigfem_b200 import capi
    P = capi.Problem(capi.ProblemDesc(**spec_kwargs(CASES["coh_op"])))
    dU = torch.zeros(P.n_nodes * P.dim, dtype=torch.float64, device="cuda")
    f = torch.zeros(P.n_free, dtype=torch.float64, device="cuda")
    p = torch.zeros(max(1, P.n_const), dtype=torch.float64, device="cuda")
    with pytest.raises(capi.PigfemError) as e:
        P.material_sensitivity(dU.data_ptr(), 0, 0, f.data_ptr(), p.data_ptr())
    assert e.value.code == 4
    with pytest.raises(capi.PigfemError) as e:
        P.material_sensitivity(dU.data_ptr(), 2, 0, f.data_ptr(), p.data_ptr())
    assert e.value.code == 2
    P.close()
