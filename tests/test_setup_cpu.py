"""CPU tests (no GPU): the C ABI library, the host set-up against the reference, and the pinning
of the golden fixtures.

* libpigfem_b200.so loads and exports every function include/pigfem_b200.h declares;
* the host IGFEM set-up (pg_create_host: detection, enrichment nodes, sub-element quadrature,
  DOF numbering, CSR preallocation) reproduces the reference's enriched mesh: coordinates and
  DOF numbers bit-exact, CSR patterns of K_ff/K_fp/K_pf/K_pp bit-exact, and -- against the
  live reference -- the sub-element and cohesive quadrature data to 1e-13;
* the committed fixtures are what the reference computes today (regenerated bit-exact);
* set-up errors come back as status codes, never as exits.
"""
import ctypes
import os
import re

import numpy as np
import pytest

from tests.conftest import ROOT
from tests.golden.cases import CASES, spec_kwargs

GOLDEN = os.path.join(ROOT, "tests", "golden")
HEADER = os.path.join(ROOT, "include", "pigfem_b200.h")
DROPIN_HEADER = os.path.join(ROOT, "include", "pigfem_b200_dropin.h")


def header_functions(path=HEADER):
    txt = open(path).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?(?:int|void|char\s*\*|const char\s*\*)\s*\*?\s*(pg_\w+)\s*\(", txt, flags=re.M)))


def host_problem(name):
    from pigfem_b200 import capi
    return capi.Problem(capi.ProblemDesc(**spec_kwargs(CASES[name])), device=False)


def test_library_exports_every_declared_function():
    from pigfem_b200 import capi
    L = capi.load_library()
    names = header_functions()
    assert len(names) >= 20, names
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert set(capi.EXPORTED) <= set(names)


def test_dropin_build_exports_its_binding_calls():
    """The reference built with the drop-in Assembler::assemble (oracle/_ref/libpigfem_ref_b200.so)
    exports every call include/pigfem_b200_dropin.h declares, and its Assembler::assemble is the
    drop-in's (the reference's own definition is weak in that build)."""
    from oracle import ref
    if not ref.available("b200"):
        pytest.skip("drop-in variant of the oracle not built")
    L = ctypes.CDLL(ref.LIB_B200_PATH)
    names = header_functions(DROPIN_HEADER)
    assert names == ["pg_dropin_bind", "pg_dropin_last_error", "pg_dropin_unbind"], names
    assert all(hasattr(L, n) for n in names)


@pytest.mark.parametrize("name", sorted(CASES))
def test_host_setup_matches_golden(name):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    P = host_problem(name)
    X, dofs, _ = P.nodes()
    dim = P.dim
    Xr = np.concatenate([g["node_coords"], g["enrich_coords"]]).reshape(-1, dim)
    assert X.shape == Xr.shape
    assert np.array_equal(X, Xr), np.abs(X - Xr).max()
    assert np.array_equal(dofs.reshape(-1), g["node_dofs"])
    for b, key in enumerate(("K_ff", "K_fp", "K_pf", "K_pp")):
        rp, ci, _ = P.pattern(b)
        assert np.array_equal(rp, g[key + "_rowptr"]), key
        assert np.array_equal(ci, g[key + "_cols"]), key
    assert P.n_isv == len(g["isv_committed"])
    P.close()


@pytest.mark.parametrize("name", ["lin_tri3_three_fibers", "lin_tri3_polygon", "coh_bl_polygon", "coh_bl",
                                  "coh_xn", "coh_bl_two_fibers_one_element", "lin_tet4_one_sphere", "coh_tet4_bl",
                                  "coh_tet4_opaug_two_spheres", "lin_quad4_one_fiber", "lin_quad4_fiber_subscale",
                                  "coh_quad4_bl", "coh_quad4_bl_two_fibers_one_element"])
def test_host_quadrature_matches_live_reference(oracle_lib, name):
    ref = oracle_lib
    R = ref.RefProblem(ref.ProblemSpec(**spec_kwargs(CASES[name])))
    P = host_problem(name)
    ecut, qoff = R.get("elem_cut"), R.get("elem_qp_off")
    J, W, goff, grad = R.get("qp_J"), R.get("qp_W"), R.get("qp_grad_off"), R.get("qp_grad")
    cut_elem, cqoff = P.debug("cut_elem"), P.debug("cut_qp_off")
    wgt, pgoff, pgrad = P.debug("qp_wgt"), P.debug("qp_grad_off"), P.debug("qp_grad")
    assert np.array_equal(np.nonzero(ecut)[0], cut_elem)
    for c, e in enumerate(cut_elem):
        rw = J[qoff[e]:qoff[e + 1]] * W[qoff[e]:qoff[e + 1]]
        pw = wgt[cqoff[c]:cqoff[c + 1]]
        assert len(rw) == len(pw), e
        assert np.abs(rw - pw).max() <= 1e-13 * np.abs(rw).max(), e
        rg = grad[goff[qoff[e]]:goff[qoff[e + 1]]]
        pg = pgrad[pgoff[cqoff[c]]:pgoff[cqoff[c + 1]]]
        assert len(rg) == len(pg), e
        assert np.abs(rg - pg).max() <= 1e-13 * np.abs(rg).max(), e
    if CASES[name]["coh_law"]:
        assert np.array_equal(R.get("coh_struct"), P.debug("coh_local"))
        cN, cR, cJ, cW = R.get("coh_qp_N"), R.get("coh_qp_R"), R.get("coh_qp_J"), R.get("coh_qp_W")
        assert np.abs(cN - P.debug("cqp_N")).max() <= 1e-14
        assert np.abs(cR - P.debug("cqp_R")).max() <= 1e-14
        assert np.abs(cJ * cW - P.debug("cqp_wgt")).max() <= 1e-14 * np.abs(cJ * cW).max()
    P.close()
    R.close()


@pytest.mark.parametrize("name", ["lin_tri3_one_fiber", "lin_tri3_subscale", "coh_bl", "coh_opaug", "coh_xn",
                                  "coh_bl_two_fibers_one_element", "lin_tet4_subscale", "coh_tet4_xn",
                                  "coh_quad4_bl_two_fibers_one_element"])
def test_golden_fixtures_reproduce(oracle_lib, name):
    """The reference, built here from its sources, regenerates the committed fixture bit-exactly."""
    from tests.golden import make_golden
    out, _ = make_golden.generate(name)
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    assert sorted(out) == sorted(g.files)
    for k in g.files:
        assert np.array_equal(out[k], g[k]), k


@pytest.mark.parametrize("name", ["lin_tri3_plies", "coh_bl_plies", "lin_tet4_plies", "lin_tri3_ply_cut", "coh_bl_ply_cut",
                                  "lin_tet4_ply_cut", "coh_tet4_bl_ply_cut", "lin_tri3_three_fibers"])
def test_element_materials_match_live_reference(oracle_lib, name):
    """Every uncut element and every sub-element quadrature point carries the reference's material:
    matrix, fiber, or -- in the bounding plies (every node in the top or bottom fraction of the
    height) -- the transversely isotropic ply material, which the matrix side of a cut ply element
    keeps."""
    ref = oracle_lib
    R = ref.RefProblem(ref.ProblemSpec(**spec_kwargs(CASES[name])))
    P = host_problem(name)
    ecut, qoff, qmat = R.get("elem_cut"), R.get("elem_qp_off"), R.get("qp_mat")
    mats = R.get("materials").reshape(-1, 3)
    # reference material index -> 0 matrix, 1 fiber, 2 ply
    code = np.where(mats[:, 0] == 2, 2, np.where(mats[:, 1] == spec_kwargs(CASES[name])["E_fiber"], 1, 0))
    uncut = np.nonzero(ecut == 0)[0]
    ref_mat = code[qmat[qoff[uncut]]]
    mine = P.debug("elem_mat")[uncut]
    assert np.array_equal(mine, ref_mat)
    # the sub-element quadrature points of the cut elements, in the reference's order
    cut = np.nonzero(ecut)[0]
    ref_qp = code[np.concatenate([qmat[qoff[e]:qoff[e + 1]] for e in cut])] if len(cut) else np.zeros(0)
    assert np.array_equal(P.debug("qp_mat"), ref_qp)
    if CASES[name].get("ply_frac", 0.0) > 0:
        assert (mine == 2).sum() > 0 and (mine == 1).sum() > 0
        if CASES[name].get("ply_cut"):
            assert (ref_qp == 2).sum() > 0 and (ref_qp == 1).sum() > 0
    P.close()
    R.close()


def test_setup_errors_are_status_codes():
    from pigfem_b200 import capi
    # a mesh node exactly on a fiber surface (x = 0.5, y = 0.25 on an 8 x 8 grid)
    with pytest.raises(capi.PigfemError) as e:
        capi.Problem(capi.ProblemDesc(n=(8, 8), inclusions=np.array([[0.5, 0.5, 0.25]])), device=False)
    assert e.value.code == 3
    # invalid descriptions
    with pytest.raises(capi.PigfemError) as e:
        capi.Problem(capi.ProblemDesc(n=(0, 8)), device=False)
    assert e.value.code == 2
    with pytest.raises(capi.PigfemError) as e:
        capi.Problem(capi.ProblemDesc(n=(8, 8), inclusions=np.array([[0.5, 0.5, -0.1]])), device=False)
    assert e.value.code == 2
    # an unknown cohesive law, and trilinear parameters out of order (the reference's setters stop there)
    with pytest.raises(capi.PigfemError) as e:
        capi.Problem(capi.ProblemDesc(n=(8, 8), coh_law=13, coh=(50.0, 1e-6, 1e-3, 5e-3)), device=False)
    assert e.value.code == 2
    with pytest.raises(capi.PigfemError) as e:
        capi.Problem(capi.ProblemDesc(n=(8, 8), coh_law=capi.COH_TL, coh=(50.0, 1e-3, 5e-7, 5e-3)), device=False)
    assert e.value.code == 2
    # bounding plies: a ply fraction of half the height or more, and a ply material with a
    # non-positive modulus
    ply = (36.2e3, 7.11e3, 2.32e3, 2.17e3, 0.335)
    with pytest.raises(capi.PigfemError) as e:
        capi.Problem(capi.ProblemDesc(n=(8, 8), ply_frac=0.5, ply=ply), device=False)
    assert e.value.code == 2
    with pytest.raises(capi.PigfemError) as e:
        capi.Problem(capi.ProblemDesc(n=(8, 8), ply_frac=0.25, ply=(36.2e3, 0.0, 2.32e3, 2.17e3, 0.335)), device=False)
    assert e.value.code == 2


def test_uncut_sizes():
    """An uncut 4 x 4 tri3 mesh: 25 nodes, 32 elements, Dirichlet left/right columns."""
    from pigfem_b200 import capi
    P = capi.Problem(capi.ProblemDesc(n=(4, 4)), device=False)
    s = P.sizes
    assert (s["n_nodes"], s["n_elem"], s["n_cut_elem"], s["n_enrich_nodes"]) == (25, 32, 0, 0)
    # left column u_x = 0 (5 dofs), right column u_x prescribed (5 dofs), node 0 also u_y = 0
    assert s["n_const"] == 11 and s["n_free"] == 39
    P.close()


def test_device_entry_points_refuse_host_only_contexts():
    """A context built by the host set-up alone (no pg_upload) has no device tables: every entry
    point that launches work returns PG_ERR_STATE before touching the GPU."""
    import ctypes
    from pigfem_b200 import capi
    L = capi.load_library()
    P = host_problem("lin_tri3_subscale")
    h = P.h
    buf = np.zeros(64)
    dptr = ctypes.c_void_p(4096)   # never dereferenced: the residency check comes first
    eps = np.zeros(6)
    out = ctypes.c_double(0.0)
    assert L.pg_assemble_device(h, dptr, 1.0, capi.FUNC | capi.JAC) == 12
    assert L.pg_residual_strains(h, dptr, 1.0, 1, eps.ctypes.data, dptr, dptr) == 12
    assert L.pg_assemble(h, buf.ctypes.data, 1.0, capi.FUNC, None, None, None, None, buf.ctypes.data, buf.ctypes.data) == 12
    assert L.pg_residual_norm(h, ctypes.byref(out)) == 12
    assert L.pg_homogenize(h, dptr, 1.0, buf.ctypes.data) == 12
    it = np.zeros(1, np.int32)
    assert L.pg_pcg_solve(h, dptr, dptr, 1, 1e-8, 10, it.ctypes.data, buf.ctypes.data) == 12
    P.close()
