"""Batched assembly (pg_batch_*): many contexts in one set of persistent launches replayed from a
CUDA graph give, for every context, bitwise the K values, residual, trial internal variables and
damage zones of that context assembled alone -- in FP64 and FP32-mixed, before and after the
autotuner changes the launch shape, in 2D and 3D."""
import os

import numpy as np
import pytest

from tests.golden.cases import CASES, cohesive_state, spec_kwargs

pytestmark = pytest.mark.gpu


def _outputs(P):
    from pigfem_b200 import capi
    import torch
    torch.cuda.synchronize()
    K4, pf, pp = P.device_outputs()
    out = {}
    for b, key in enumerate(("K_ff", "K_fp", "K_pf", "K_pp")):
        out[key] = capi.device_view(K4[b], P.nnz[b]).cpu().numpy().copy() if P.nnz[b] else np.zeros(0)
    out["P_f"] = capi.device_view(pf, P.n_free).cpu().numpy().copy()
    out["P_p"] = capi.device_view(pp, P.n_const).cpu().numpy().copy() if P.n_const else np.zeros(0)
    if P.n_isv:
        out["isv"] = P.get_isv(True)
        out["zones"] = P.damage_zones()
    return out


def _problems(names, extra_2d=0):
    import torch
    from pigfem_b200 import capi, rve
    probs, us = [], []
    for name in names:
        g = np.load(os.path.join(os.path.dirname(__file__), "golden", name + ".npz"))
        P = capi.Problem(capi.ProblemDesc(**spec_kwargs(CASES[name])))
        if P.n_isv:
            P.set_isv(g["isv_committed"])
        probs.append(P)
        us.append(torch.from_numpy(g["U_dof"][g["node_dofs"]]).cuda())
    for k in range(extra_2d):
        R = rve.cohesive_2d(n=48 + 16 * k, n_fibers=6 + 3 * k, r_lo=0.04, r_hi=0.07, gap=0.01, request=k)
        P = capi.Problem(R.desc)
        probs.append(P)
        us.append(torch.from_numpy(rve.interface_state(P, seed=k)).cuda())
    return probs, us


def _check_batch(probs, us, flags, tune=False):
    from pigfem_b200 import capi
    alone = []
    for P, u in zip(probs, us):
        P.assemble_device(u.data_ptr(), 1.0, flags)
        alone.append(_outputs(P))
    B = capi.Batch(probs)
    ptrs = [u.data_ptr() for u in us]
    if tune:
        shape = B.tune(ptrs, flags, reps=1)
        assert all(s > 0 for s in shape)
    for rep in range(2):          # two replays of the same graph
        B.assemble(ptrs, flags)
        B.wait()
        for i, P in enumerate(probs):
            got = _outputs(P)
            for k in alone[i]:
                assert np.array_equal(got[k], alone[i][k]), (i, k, rep)
    B.close()


@pytest.mark.parametrize("fp32", [False, True], ids=["fp64", "fp32_mixed"])
def test_batch_2d_bitwise_equals_alone(fp32):
    from pigfem_b200 import capi
    probs, us = _problems(["coh_bl", "coh_xn", "lin_tri3_three_fibers", "coh_bl_polygon", "lin_tri3_subscale", "coh_stl",
                           "coh_tlnu_compression"], extra_2d=3)
    flags = capi.FUNC | capi.JAC | (capi.FP32 if fp32 else 0)
    _check_batch(probs, us, flags)
    for P in probs:
        P.close()


def test_batch_autotuned_shape_keeps_results():
    from pigfem_b200 import capi
    probs, us = _problems(["coh_opaug", "coh_bl_two_fibers_one_element"], extra_2d=2)
    _check_batch(probs, us, capi.FUNC | capi.JAC | capi.FP32, tune=True)
    for P in probs:
        P.close()


def test_batch_3d_bitwise_equals_alone():
    from pigfem_b200 import capi
    probs, us = _problems(["coh_tet4_bl", "coh_tet4_opaug_two_spheres", "lin_tet4_subscale", "lin_tet4_uncut", "coh_tet4_tl"])
    _check_batch(probs, us, capi.FUNC | capi.JAC)
    for P in probs:
        P.close()


def test_batch_rejects_mixed_dimensions():
    from pigfem_b200 import capi
    probs, _ = _problems(["coh_bl", "lin_tet4_uncut"])
    with pytest.raises(capi.PigfemError):
        capi.Batch(probs)
    for P in probs:
        P.close()


def test_batch_3d_autotuned_shape_keeps_results():
    """3D: the shape the autotuner picks (persistent blocks per SM among 2, 4, 8, 16) leaves every
    context's results bitwise those of the single-context call."""
    from pigfem_b200 import capi
    probs, us = _problems(["coh_tet4_opaug_two_spheres", "lin_tet4_one_sphere", "coh_tet4_tl"])
    _check_batch(probs, us, capi.FUNC | capi.JAC, tune=True)
    for P in probs:
        P.close()
