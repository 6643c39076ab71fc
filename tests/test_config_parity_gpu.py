"""GPU parity at the benchmarked configurations, against the reference's own assembly run live.

The three single-RVE workloads are assembled through the C ABI and by the reference's
Assembler::assemble (oracle/_ref, compiled from the reference's sources) on the same mesh,
displacement state and committed internal variables:

  * 2D linear, 64 x 64 quads split into 8,192 tri3, ten fibers r ~ U[0.03, 0.06], gap 0.01,
    1 % strain prescribed on the right edge;
  * 2D cohesive, 512 x 512 quads split into 524,288 tri3, 200 fibers r ~ U[0.008, 0.015],
    gap 0.002, bilinear interfaces, a state whose openings run through the law's loading,
    softening and failed branches;
  * 3D linear, 64^3 hexes split into 1,572,864 tet4, 50 spheres r ~ U[0.04, 0.08], gap 0.01,
    periodic, K with the first unit strain and the residuals of all six unit strains.

Bar: the DOF numbering, the four CSR patterns and the damage zones bit-exact; K values, P_f, P_p
and the trial internal variables within 1e-12 relative Frobenius error (FP64).  The FP32-mixed
path is held to 1e-5 on K and R, and its measured errors are printed (pytest -s shows them).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
FP32_TOL = 1e-5
BLOCKS = ("K_ff", "K_fp", "K_pf", "K_pp")


def rel(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def spec_of(ref, desc):
    import dataclasses
    return ref.ProblemSpec(**{f.name: getattr(desc, f.name) for f in dataclasses.fields(desc)})


def check_structure(P, R):
    _, dofs, _ = P.nodes()
    assert np.array_equal(dofs.reshape(-1), R.get("node_dofs")), "DOF numbering differs"
    for b, key in enumerate(BLOCKS):
        rp, ci, _, _ = R.csr(key)
        prp, pci, _ = P.pattern(b)
        assert np.array_equal(rp, prp) and np.array_equal(ci, pci), key + " pattern"


def compare(out, R, tol):
    errs = {key: rel(out[key], R.csr(key)[2]) for key in BLOCKS}
    errs["P_f"] = rel(out["P_f"], R.get("P_f"))
    errs["P_p"] = rel(out["P_p"], R.get("P_p"))
    bad = {k: v for k, v in errs.items() if not v <= tol}
    assert not bad, bad
    return errs


def test_linear_2d_64(oracle_lib):
    """64 x 64 tri3, ten fibers, 1 % strain: one K and R assembly."""
    from pigfem_b200 import capi, rve
    ref = oracle_lib
    W = rve.linear_2d()
    assert len(W.fibers) == 10
    R = ref.RefProblem(spec_of(ref, W.desc))
    P = capi.Problem(W.desc)
    assert P.sizes["n_elem"] == 8192 and P.sizes["n_cut_elem"] > 0
    # a displacement near the loaded state: the prescribed values on the constrained DOFs, small
    # seeded values on the free ones
    _, dofs, dirichlet = P.nodes()
    rng = np.random.default_rng(64)
    Ud = np.concatenate([rng.uniform(-1e-3, 1e-3, R.n_free), dirichlet])
    R.assemble(Ud, None, 1.0)
    check_structure(P, R)
    U = Ud[dofs.reshape(-1)]
    e64 = compare(P.assemble(U, 1.0), R, FP64_TOL)
    e32 = compare(P.assemble(U, 1.0, flags=capi.FUNC | capi.JAC | capi.FP32), R, FP32_TOL)
    print(f"\nlinear_2d_64 FP64 errors {e64}\nlinear_2d_64 FP32-mixed errors {e32}")
    R.close()
    P.close()


@pytest.fixture(scope="module")
def cohesive_512(oracle_lib):
    from pigfem_b200 import capi, rve
    ref = oracle_lib
    W = rve.cohesive_2d()
    R = ref.RefProblem(spec_of(ref, W.desc))
    P = capi.Problem(W.desc)
    yield W, R, P
    R.close()
    P.close()


def test_cohesive_2d_512_state_from_either_mesh(cohesive_512):
    """The benchmark state built from the reference's mesh tables equals the one built from this
    library's set-up tables (the two arms of bench.py time the same state)."""
    from pigfem_b200 import rve
    W, R, P = cohesive_512
    a = rve.interface_state(P, seed=0)
    b = rve.interface_state_tables(**R.cut_tables(), seed=0)
    assert a.shape == b.shape
    assert rel(a, b) <= 1e-14


def test_cohesive_2d_512(cohesive_512):
    """512 x 512 tri3, 200 fibers, bilinear interfaces: the bench state, FP64 and FP32-mixed."""
    from pigfem_b200 import capi, rve
    W, R, P = cohesive_512
    assert P.sizes["n_elem"] == 524288 and len(W.fibers) == 200
    U = rve.interface_state_tables(**R.cut_tables(), seed=0)
    _, dofs, _ = P.nodes()
    Ud = np.zeros(R.n_free + R.n_const)
    Ud[dofs.reshape(-1)] = U
    isv = np.zeros(P.n_isv)
    R.assemble(Ud, isv, 1.0)
    check_structure(P, R)
    P.set_isv(isv)
    e64 = compare(P.assemble(U, 1.0), R, FP64_TOL)
    assert rel(P.get_isv(True), R.get("isv_trial")) <= FP64_TOL
    zones = P.damage_zones()
    assert np.array_equal(zones, R.get("coh_zone").astype(np.uint8))
    # the state exercises the loading, softening and failed branches
    assert {1, 2, 3} <= set(np.unique(zones).tolist()), np.unique(zones)
    e32 = compare(P.assemble(U, 1.0, flags=capi.FUNC | capi.JAC | capi.FP32), R, FP32_TOL)
    assert np.array_equal(P.damage_zones(), zones)
    print(f"\ncohesive_2d_512 FP64 errors {e64}\ncohesive_2d_512 FP32-mixed errors {e32}")


def test_cohesive_2d_512_residual_only(cohesive_512):
    """A residual-only assembly (the Newton residual between tangents) at configuration scale."""
    from pigfem_b200 import capi, rve
    W, R, P = cohesive_512
    U = rve.interface_state_tables(**R.cut_tables(), seed=3, open_hi=2e-3)
    _, dofs, _ = P.nodes()
    Ud = np.zeros(R.n_free + R.n_const)
    Ud[dofs.reshape(-1)] = U
    isv = np.zeros(P.n_isv)
    R.assemble(Ud, isv, 1.0, func=True, jac=False)
    P.set_isv(isv)
    out = P.assemble(U, 1.0, flags=capi.FUNC)
    assert rel(out["P_f"], R.get("P_f")) <= FP64_TOL
    assert rel(out["P_p"], R.get("P_p")) <= FP64_TOL
    assert np.array_equal(P.damage_zones(), R.get("coh_zone").astype(np.uint8))


def test_linear_3d_64(oracle_lib):
    """64^3 tet4, 50 spheres, periodic: K and R with the first unit strain, then the residuals of
    the other five unit strains from one multi-strain pass, each against the reference's
    residual-only assembly with that strain."""
    import torch
    from pigfem_b200 import capi, rve
    ref = oracle_lib
    W = rve.linear_3d()
    assert len(W.fibers) == 50
    R = ref.RefProblem(spec_of(ref, W.desc))
    P = capi.Problem(W.desc)
    assert P.sizes["n_elem"] == 1572864 and P.sizes["n_cut_elem"] > 0
    rng = np.random.default_rng(643)
    Ud = rng.uniform(-1e-3, 1e-3, R.n_free + R.n_const)
    _, dofs, _ = P.nodes()
    U = Ud[dofs.reshape(-1)]
    strains = [tuple(1.0 if i == k else 0.0 for i in range(6)) for k in range(6)]
    R.set_macro(strains[0])
    R.assemble(Ud, None, 1.0)
    check_structure(P, R)
    P.set_macro_strain(strains[0])
    e64 = compare(P.assemble(U, 1.0), R, FP64_TOL)
    e32 = compare(P.assemble(U, 1.0, flags=capi.FUNC | capi.JAC | capi.FP32), R, FP32_TOL)
    print(f"\nlinear_3d_64 FP64 errors {e64}\nlinear_3d_64 FP32-mixed errors {e32}")
    dU = torch.from_numpy(np.ascontiguousarray(U)).cuda()
    nf, nc = P.n_free, P.n_const
    Rf = torch.full((5 * nf,), float("nan"), dtype=torch.float64, device="cuda")
    Rp = torch.full((max(1, 5 * nc),), float("nan"), dtype=torch.float64, device="cuda")
    P.residual_strains(dU.data_ptr(), strains[1:], Rf.data_ptr(), Rp.data_ptr() if nc else 0, 1.0)
    torch.cuda.synchronize()
    Rf = Rf.cpu().numpy()
    Rp = Rp.cpu().numpy()
    for k in range(1, 6):
        R.set_macro(strains[k])
        R.assemble(Ud, None, 1.0, func=True, jac=False)
        assert rel(Rf[(k - 1) * nf:k * nf], R.get("P_f")) <= FP64_TOL, k
        if nc:
            assert rel(Rp[(k - 1) * nc:k * nc], R.get("P_p")) <= FP64_TOL, k
    R.close()
    P.close()
