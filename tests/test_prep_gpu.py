"""Device IGFEM preprocessing (pg_create_prep_device) against the host set-up (pg_create_host).

The device passes -- node detection, the element pass of the cut detection, the enrichment nodes
with their intersection points, the standard nodes' DOF numbering, and (PG_PREP_PATTERN) the DOF
nodes' adjacency and the CSR pattern -- replace the host's own loops, so every table of the two
set-ups must agree: integer tables (detection values, element
materials, cut elements, enrichment edges, sub-element and cohesive topology, DOF numbers, the
four CSR patterns) bit-exact, and the coordinates and quadrature data too (the device passes are
compiled without floating-point contraction and form every value with the host's operations).
Cases: every golden case (tri3 / quad4 / tet4, cohesive and linear, Dirichlet and periodic,
plies, two inclusions in one element) and the three benchmarked single-RVE meshes.
"""
import numpy as np
import pytest

from tests.golden.cases import CASES, spec_kwargs

pytestmark = pytest.mark.gpu

TABLES = ("node_detect", "elem_mat", "cut_of", "cut_elem", "enr_edge", "enr_incl", "conn", "cut_node_off",
          "cut_nodes", "sub_type", "cut_sub_off", "sub_mat", "cut_qp_off", "qp_wgt", "qp_mat", "qp_grad_off",
          "qp_grad", "cut_coh_off", "coh_nh", "coh_local_off", "coh_local", "coh_qp_off", "cqp_N", "cqp_R",
          "cqp_wgt", "cqp_isv", "dn_node", "dn_nbr_off", "dn_nbr", "dn_adj_off", "dn_adj")


def both(desc, pattern=True):
    from pigfem_b200 import capi
    H = capi.Problem(desc, device=False)
    D = capi.Problem(desc, device=False, prep_device=True, prep_pattern=pattern)
    return H, D


def assert_same_setup(H, D):
    assert H.sizes == D.sizes
    for name in TABLES:
        a, b = H.debug(name), D.debug(name)
        assert a.dtype == b.dtype and a.shape == b.shape, name
        assert np.array_equal(a, b), name
    for blk in range(4):
        for x, y in zip(H.pattern(blk), D.pattern(blk)):
            if isinstance(x, np.ndarray):
                assert np.array_equal(x, y), blk
            else:
                assert x == y
    XH, dH, pH = H.nodes()
    XD, dD, pD = D.nodes()
    assert np.array_equal(dH, dD)
    assert np.array_equal(XH, XD)
    assert np.array_equal(pH, pD)


@pytest.mark.parametrize("name", sorted(CASES))
def test_device_prep_matches_host_setup(name):
    from pigfem_b200 import capi
    H, D = both(capi.ProblemDesc(**spec_kwargs(CASES[name])))
    assert_same_setup(H, D)
    # the per-node passes alone (PG_PREP_NODES, the pattern on the host threads)
    _, D1 = both(capi.ProblemDesc(**spec_kwargs(CASES[name])), pattern=False)
    assert_same_setup(H, D1)
    n = CASES[name]["n"]
    if min(n) >= 2:
        assert D.prep_device_ms() >= 0.0
    assert H.prep_device_ms() == -1.0


def test_device_prep_benchmark_meshes():
    from pigfem_b200 import rve
    for r in (rve.linear_2d(64, 10), rve.cohesive_2d(512, 200), rve.linear_3d(64, 50)):
        H, D = both(r.desc)
        assert_same_setup(H, D)
        print(f"{r.desc.n}: device passes {D.prep_device_ms():.3f} ms, {D.sizes['n_enrich_nodes']} enrichment nodes")


def test_device_prep_reports_surface_node_like_the_host():
    from pigfem_b200 import capi
    desc = capi.ProblemDesc(n=(8, 8), inclusions=np.array([[0.5, 0.5, 0.25]]))
    msgs = []
    for prep in (False, True):
        with pytest.raises(capi.PigfemError) as e:
            capi.Problem(desc, device=False, prep_device=prep)
        assert e.value.code == 3
        msgs.append(str(e.value))
    assert msgs[0] == msgs[1]


def test_device_prep_assembles_like_the_host():
    """The device-prepared context uploads and assembles to the host-prepared one's values."""
    import os
    from pigfem_b200 import capi
    from tests.conftest import ROOT
    g = np.load(os.path.join(ROOT, "tests", "golden", "coh_bl.npz"))
    H, D = both(capi.ProblemDesc(**spec_kwargs(CASES["coh_bl"])))
    H.upload()
    D.upload()
    U = g["U_dof"][g["node_dofs"]]
    for P in (H, D):
        P.set_isv(g["isv_committed"])
    a, b = H.assemble(U, 1.0), D.assemble(U, 1.0)
    for k in ("K_ff", "K_fp", "K_pf", "K_pp", "P_f", "P_p"):
        assert np.array_equal(a[k], b[k]), k
