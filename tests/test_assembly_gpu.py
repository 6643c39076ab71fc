"""GPU parity of the assembly path against the reference's own CPU assembly.

Each case of tests/golden/cases.py is assembled through the C ABI (libpigfem_b200.so, sm_100a
kernels) and compared with the reference's Assembler::assemble output stored in
tests/golden/<case>.npz (generated by tests/golden/make_golden.py from oracle/_ref):
  * CSR pattern of K_ff / K_fp / K_pf / K_pp: bit-exact;
  * K values and the internal-force parts P_f / P_p: relative Frobenius error <= 1e-12 (FP64);
  * trial internal variables: relative error <= 1e-12;
  * cohesive damage zones: bit-exact.
The FP32-mixed path is held to 1e-5 relative error on K and R.
"""
import os

import numpy as np
import pytest

from tests.conftest import ROOT
from tests.golden.cases import CASES, spec_kwargs

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(ROOT, "tests", "golden")
FP64_TOL = 1e-12
FP32_TOL = 1e-5


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def row_rel(vals, ref_vals, rowptr):
    """max over rows of max|a - b| / max|b| within the row: entries that do not share a row with a
    stiff contribution (a compression penalty, a fiber) are still held to the tolerance.  The row
    scale is floored at 1e-4 of the block's largest entry, so with the 1e-11 bound an entry is
    never held tighter than 1e-15 of the block: a row whose only nonzero is the rounding residue
    of a cancelling sum (2.3e-13 in a 2.7e4 block, where the exact value is 0 and either side may
    round to 0) is judged at that scale."""
    worst = 0.0
    floor = 1e-4 * (np.abs(ref_vals).max() if len(ref_vals) else 0.0)
    for r in range(len(rowptr) - 1):
        a, b = vals[rowptr[r]:rowptr[r + 1]], ref_vals[rowptr[r]:rowptr[r + 1]]
        if len(b) == 0:
            continue
        m = max(np.abs(b).max(), floor)
        if m > 0:
            worst = max(worst, np.abs(a - b).max() / m)
    return worst


def load_case(name):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    return {k: g[k] for k in g.files}


def build(name):
    from pigfem_b200 import capi
    return capi.Problem(capi.ProblemDesc(**spec_kwargs(CASES[name])))


@pytest.mark.parametrize("name", sorted(CASES))
def test_fp64_matches_reference(name):
    g = load_case(name)
    P = build(name)
    _, dofs, _ = P.nodes()
    assert np.array_equal(dofs.reshape(-1), g["node_dofs"]), "DOF numbering differs"
    for b, key in enumerate(("K_ff", "K_fp", "K_pf", "K_pp")):
        rp, ci, _ = P.pattern(b)
        assert np.array_equal(rp, g[key + "_rowptr"]) and np.array_equal(ci, g[key + "_cols"]), key + " pattern"
    if P.n_isv:
        P.set_isv(g["isv_committed"])
    U = g["U_dof"][g["node_dofs"]]
    out = P.assemble(U, 1.0)
    for key in ("K_ff", "K_fp", "K_pf", "K_pp"):
        assert rel(out[key], g[key + "_vals"]) <= FP64_TOL, (key, rel(out[key], g[key + "_vals"]))
        assert row_rel(out[key], g[key + "_vals"], g[key + "_rowptr"]) <= 1e-11, key
    assert rel(out["P_f"], g["P_f"]) <= FP64_TOL, rel(out["P_f"], g["P_f"])
    assert rel(out["P_p"], g["P_p"]) <= FP64_TOL, rel(out["P_p"], g["P_p"])
    if P.n_isv:
        assert rel(P.get_isv(trial=True), g["isv_trial"]) <= FP64_TOL
    if CASES[name]["coh_law"]:
        assert np.array_equal(P.damage_zones(), g["coh_zone"].astype(np.uint8))


@pytest.mark.parametrize("name", ["lin_tri3_three_fibers", "coh_bl", "lin_tri3_subscale", "lin_tet4_subscale",
                                  "coh_tet4_bl"])
def test_fp32_mixed_error_bound(name):
    from pigfem_b200 import capi
    g = load_case(name)
    P = build(name)
    if P.n_isv:
        P.set_isv(g["isv_committed"])
    U = g["U_dof"][g["node_dofs"]]
    out = P.assemble(U, 1.0, flags=capi.FUNC | capi.JAC | capi.FP32)
    for key in ("K_ff", "K_fp", "K_pf", "K_pp"):
        assert rel(out[key], g[key + "_vals"]) <= FP32_TOL, (key, rel(out[key], g[key + "_vals"]))
    assert rel(out["P_f"], g["P_f"]) <= FP32_TOL


def test_deterministic_bitwise():
    """Two assemblies of the same state are bit-identical (no atomics in the scatter)."""
    g = load_case("coh_bl")
    P = build("coh_bl")
    U = g["U_dof"][g["node_dofs"]]
    a = {k: v.copy() for k, v in P.assemble(U).items()}
    b = P.assemble(U)
    for k in a:
        assert np.array_equal(a[k], b[k]), k


@pytest.mark.parametrize("name", ["coh_op", "lin_tri3_subscale", "coh_bl_polygon", "lin_tet4_subscale",
                                  "coh_tet4_opaug_two_spheres", "lin_quad4_subscale", "coh_quad4_op"])
def test_func_only_and_jac_only(name):
    """A residual-only assembly (the residual-only kernels) gives the residual of a full one to
    1e-14 and bitwise its trial internal variables and damage zones (the cohesive kernel is the
    same), and leaves K as the last JAC assembly left it; a JAC-only assembly gives the
    reference's K.  The residual sums are the same operations in the same order; only the
    compiler's choice of which products to fuse into multiply-adds differs between the two
    kernels (built with -fmad=false the two residuals agree bitwise in all these cases)."""
    from pigfem_b200 import capi
    g = load_case(name)
    P = build(name)
    if P.n_isv:
        P.set_isv(g["isv_committed"])
    U = g["U_dof"][g["node_dofs"]]
    full = {k: v.copy() for k, v in P.assemble(U, 1.0, flags=capi.FUNC | capi.JAC).items()}
    isv_full = P.get_isv(True).copy() if P.n_isv else None
    zones_full = P.damage_zones().copy()
    assert rel(full["P_f"], g["P_f"]) <= FP64_TOL
    zero = np.zeros_like(U)
    P.assemble(zero, 1.0, flags=capi.JAC)             # K of another state in the CSR
    k_other = P.assemble(zero, 1.0, flags=capi.JAC)["K_ff"].copy()
    r = P.assemble(U, 1.0, flags=capi.FUNC)
    assert rel(r["P_f"], full["P_f"]) <= 1e-14 and rel(r["P_p"], full["P_p"]) <= 1e-14
    assert rel(r["P_f"], g["P_f"]) <= FP64_TOL
    import torch
    torch.cuda.synchronize()
    K4, _, _ = P.device_outputs()                      # untouched by the residual-only kernels
    assert np.array_equal(capi.device_view(K4[0], P.nnz[0]).cpu().numpy(), k_other)
    if P.n_isv:
        assert np.array_equal(P.get_isv(True), isv_full)
    assert np.array_equal(P.damage_zones(), zones_full)
    k = P.assemble(U, 1.0, flags=capi.JAC)
    assert rel(k["K_ff"], g["K_ff_vals"]) <= FP64_TOL


def test_live_oracle_random_state(oracle_lib):
    """A fresh random state checked against the reference run live (oracle/_ref)."""
    ref = oracle_lib
    c = dict(CASES["coh_opaug"])
    R = ref.RefProblem(ref.ProblemSpec(**spec_kwargs(c)))
    P = build("coh_opaug")
    rng = np.random.default_rng(1234)
    U = rng.uniform(-3e-4, 3e-4, R.n_free + R.n_const)
    isv = rng.uniform(0, 4e-4, P.n_isv)
    R.assemble(U, isv, 1.0)
    P.set_isv(isv)
    out = P.assemble(U[R.get("node_dofs")], 1.0)
    assert rel(out["K_ff"], R.csr("K_ff")[2]) <= FP64_TOL
    assert rel(out["P_f"], R.get("P_f")) <= FP64_TOL
    assert rel(P.get_isv(True), R.get("isv_trial")) <= FP64_TOL
    assert np.array_equal(P.damage_zones(), R.get("coh_zone").astype(np.uint8))


@pytest.mark.parametrize("kw", [
    # uncut tet4 large enough for the structured stencil rows (interior nodes 2..n-2)
    dict(elem_type=2, n=(8, 8, 8), incl=np.zeros((0, 4)), coh_law=0, coh=(0, 0, 0, 0), subscale=0, seed=31, u_scale=1e-3),
    # two cohesive spheres in a 10^3 tet mesh: stencil, general and cut rows together
    dict(elem_type=2, n=(10, 10, 10), incl=[[0.3, 0.31, 0.33, 0.17], [0.68, 0.64, 0.62, 0.2]], coh_law=7,
         coh=(50.0, 2e-4, 1.0, 0.0), subscale=0, seed=32, u_scale=1e-6, open=(1e-6, 1e-3)),
    # tri3 with fibers near every boundary and a macroscale strain on a periodic mesh
    dict(elem_type=0, n=(24, 24), incl=[[0.2, 0.2, 0.12], [0.75, 0.3, 0.1], [0.5, 0.75, 0.14]], coh_law=0,
         coh=(0, 0, 0, 0), subscale=1, eps_macro=(0.01, -0.003, 0.002), seed=33, u_scale=1e-3),
], ids=["tet4_uncut_8", "tet4_coh_two_spheres_10", "tri3_subscale_24"])
def test_live_oracle_larger_meshes(oracle_lib, kw):
    """Meshes too large for committed fixtures, checked against the reference run live."""
    from tests.golden.cases import cohesive_state
    ref = oracle_lib
    c = dict(kw)
    c.setdefault("isv_scale", 0.0)
    spec = spec_kwargs(c)
    R = ref.RefProblem(ref.ProblemSpec(**spec))
    from pigfem_b200 import capi
    P = capi.Problem(capi.ProblemDesc(**spec))
    if c["coh_law"]:
        U = cohesive_state(c, R.get("node_dofs"), R.n_free, R.n_const, R.get("elem_node_off"), R.get("elem_nodes"),
                           R.get("elem_cut"), R.get("elem_coh_off"), R.get("coh_struct"), R.get("coh_struct_off"),
                           R.get("coh_qp_off"), R.get("coh_qp_R"))
    else:
        U = np.random.default_rng(c["seed"]).uniform(-c["u_scale"], c["u_scale"], R.n_free + R.n_const)
    isv = np.zeros(P.n_isv)
    R.assemble(U, isv, 1.0)
    P.set_isv(isv)
    out = P.assemble(U[R.get("node_dofs")], 1.0)
    for b, key in enumerate(("K_ff", "K_fp", "K_pf", "K_pp")):
        rp, ci, v, _ = R.csr(key)
        prp, pci, _ = P.pattern(b)
        assert np.array_equal(rp, prp) and np.array_equal(ci, pci), key
        assert rel(out[key], v) <= FP64_TOL, (key, rel(out[key], v))
    assert rel(out["P_f"], R.get("P_f")) <= FP64_TOL
    if P.n_isv:
        assert rel(P.get_isv(True), R.get("isv_trial")) <= FP64_TOL
        assert np.array_equal(P.damage_zones(), R.get("coh_zone").astype(np.uint8))
    n_stencil = len(P.debug("fast_dn"))
    assert n_stencil > 0 or c["elem_type"] == 0
    R.close()
    P.close()


@pytest.mark.parametrize("name", ["lin_tri3_subscale", "lin_tet4_subscale"])
def test_residual_strains_equal_single_strain_assemblies(name):
    """pg_residual_strains: the residuals of several macroscale strains from one pass equal, case
    by case, residual-only assemblies with each strain set alone (to 1e-14 on the free rows, 1e-13
    on the few constrained ones: the same terms in the same order, with the compiler free to fuse
    other multiply-adds), the case with the fixture's strain equals
    the reference's residual, and K is left as the last K assembly wrote it."""
    import torch
    from pigfem_b200 import capi
    g = load_case(name)
    P = build(name)
    nv = 3 if P.dim == 2 else 6
    U = torch.from_numpy(np.ascontiguousarray(g["U_dof"][g["node_dofs"]])).cuda()
    fixture_eps = list(CASES[name]["eps_macro"])
    cases = [fixture_eps] + [list(np.eye(nv)[k] * (0.5 + k)) for k in range(nv - 1)]
    P.assemble_device(U.data_ptr(), 1.0, capi.JAC)
    torch.cuda.synchronize()
    K4, pf, pp = P.device_outputs()
    k_before = capi.device_view(K4[0], P.nnz[0]).cpu().numpy().copy()
    nf, nc = P.n_free, P.n_const
    Rf = torch.full((len(cases) * nf,), float("nan"), dtype=torch.float64, device="cuda")
    Rp = torch.full((max(1, len(cases) * nc),), float("nan"), dtype=torch.float64, device="cuda")
    P.residual_strains(U.data_ptr(), cases, Rf.data_ptr(), Rp.data_ptr() if nc else 0, 0.75)
    torch.cuda.synchronize()
    assert np.array_equal(capi.device_view(K4[0], P.nnz[0]).cpu().numpy(), k_before)
    for k, e in enumerate(cases):
        P.set_macro_strain(e)
        P.assemble_device(U.data_ptr(), 0.75, capi.FUNC)
        torch.cuda.synchronize()
        ref_f = capi.device_view(pf, nf).cpu().numpy()
        got_f = Rf[k * nf:(k + 1) * nf].cpu().numpy()
        assert rel(got_f, ref_f) <= 1e-14, (k, rel(got_f, ref_f))
        if nc:
            # the few constrained rows sum terms about 100x larger than the result, so the
            # kernels' different multiply-add fusion shows at ~1e-14 there
            assert rel(Rp[k * nc:(k + 1) * nc].cpu().numpy(), capi.device_view(pp, nc).cpu().numpy()) <= 1e-13
    # the fixture's own strain at t_frac = 1 against the reference's residual
    P.residual_strains(U.data_ptr(), cases[:1], Rf.data_ptr(), Rp.data_ptr() if nc else 0, 1.0)
    torch.cuda.synchronize()
    assert rel(Rf[:nf].cpu().numpy(), g["P_f"]) <= FP64_TOL
    P.close()


def test_residual_strains_need_a_subscale_problem():
    import torch
    from pigfem_b200 import capi
    P = build("coh_bl")
    U = torch.zeros(P.n_nodes * P.dim, dtype=torch.float64, device="cuda")
    R = torch.zeros(P.n_free + P.n_const, dtype=torch.float64, device="cuda")
    with pytest.raises(capi.PigfemError):
        P.residual_strains(U.data_ptr(), [[0.01, 0.0, 0.0]], R.data_ptr(), R.data_ptr())
    P.close()


@pytest.mark.parametrize("name", ["coh_op", "coh_tet4_bl", "coh_quad4_bl", "lin_tri3_three_fibers", "lin_tet4_subscale"])
def test_keep_static_copies_back_what_changes(name):
    """PG_KEEP_STATIC: with the host K arrays of the previous call kept, a call copies back only
    the suffix of each block from pg_changing_values on, and the arrays then hold bitwise the K
    of a full copy at the new state.  Problems without cohesive elements change no K value."""
    from pigfem_b200 import capi
    g = load_case(name)
    P = build(name)
    first = P.changing_values()
    if CASES[name]["coh_law"] == 0:
        assert first == list(P.nnz)
    else:
        assert first[0] < P.nnz[0]
    if P.n_isv:
        P.set_isv(g["isv_committed"])
    U = g["U_dof"][g["node_dofs"]]
    # a proportionally larger state: every opening grows by 5 % (a random change could push the
    # bilinear law into its compression branch, whose sinh overflows at these openings)
    U2 = 1.05 * U
    keep = {f"K_{b}": np.full(max(P.nnz[i], 1), np.nan) for i, b in enumerate(("ff", "fp", "pf", "pp"))}
    keep["P_f"] = np.zeros(max(P.n_free, 1))
    keep["P_p"] = np.zeros(max(P.n_const, 1))
    flags = capi.FUNC | capi.JAC | capi.KEEP_STATIC
    P.assemble(U, 1.0, flags, out=keep)          # first call: everything
    # poison the part a keep call must rewrite, then assemble at the new state
    for i, b in enumerate(("ff", "fp", "pf", "pp")):
        keep[f"K_{b}"][first[i]:P.nnz[i]] = np.nan
    got = P.assemble(U2, 1.0, flags, out=keep)
    full = P.assemble(U2, 1.0, capi.FUNC | capi.JAC)
    for k in ("K_ff", "K_fp", "K_pf", "K_pp", "P_f", "P_p"):
        assert np.array_equal(got[k], full[k]), k
    if CASES[name]["coh_law"]:
        # the state does change K inside the copied suffix
        assert not np.array_equal(full["K_ff"], P.assemble(U, 1.0, capi.FUNC | capi.JAC)["K_ff"])
