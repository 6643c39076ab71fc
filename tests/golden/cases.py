"""Problem cases shared by the golden-fixture generator and the parity tests.

Each case is a structured background mesh with circular (2D) or spherical (3D) inclusions, the
benchmark materials and, where named, a cohesive law on every fiber/matrix interface; a seeded
displacement field (DOF vector, free then constrained) and seeded committed internal variables
drive one assembly.  In cohesive cases the '+' (mirror) enrichment nodes are displaced from their
'-' partners along the interface normal by a seeded opening drawn from `open` (log-uniform
between the two bounds, negative bounds give compression), so every law is driven through its
loading, softening, failed and (for the memory laws, with committed maxima drawn around the
current opening) unloading branches at physically sized openings; `compress` cases exercise the
compression penalty at openings where it stays finite.  Sizes are small enough for the reference's
CPU assembly to finish in well under a second.
"""
import numpy as np

E_M, NU_M, E_F, NU_F = 3.5e3, 0.35, 72e3, 0.22
BL = (50.0, 5e-7, 5e-3, 0.0)
XN = (50.0, 2e-4, 3e-4, 1.7)
OP = (50.0, 2e-4, 1.0, 0.0)
TL = (50.0, 5e-7, 1e-3, 5e-3)
# transversely isotropic bounding plies (E1, E2, G12, G23, nu12), the glass/epoxy ply of the
# reference's RVE driver
PLY = (36.2e3, 7.11e3, 2.32e3, 2.17e3, 0.335)

CASES = {
    # name: dict(elem_type, n, incl, coh_law, coh, subscale, eps_macro, u_scale, isv_scale, seed)
    "lin_tri3_one_fiber": dict(elem_type=0, n=(8, 8), incl=[[0.5, 0.5, 0.23]], coh_law=0, coh=(0, 0, 0, 0),
                               subscale=0, u_scale=1e-3, isv_scale=0.0, seed=1),
    "lin_tri3_three_fibers": dict(elem_type=0, n=(16, 16), incl=[[0.3, 0.3, 0.12], [0.63, 0.56, 0.13], [0.45, 0.78, 0.1]],
                                  coh_law=0, coh=(0, 0, 0, 0), subscale=0, u_scale=1e-3, isv_scale=0.0, seed=2),
    "lin_tri3_two_fibers_one_element": dict(elem_type=0, n=(8, 8), incl=[[0.3817, 0.5123, 0.1031], [0.6022, 0.4871, 0.1017]],
                                            coh_law=0, coh=(0, 0, 0, 0), subscale=0, u_scale=1e-3, isv_scale=0.0, seed=3),
    "lin_tri3_subscale": dict(elem_type=0, n=(12, 12), incl=[[0.41, 0.47, 0.2]], coh_law=0, coh=(0, 0, 0, 0),
                              subscale=1, eps_macro=(0.01, -0.004, 0.002), u_scale=1e-3, isv_scale=0.0, seed=4),
    "coh_bl": dict(elem_type=0, n=(16, 16), incl=[[0.3, 0.3, 0.12], [0.63, 0.56, 0.13]], coh_law=1, coh=BL,
                   subscale=0, u_scale=1e-6, isv_scale=0.0, seed=5, open=(1e-7, 1.2e-2)),
    "coh_blnu": dict(elem_type=0, n=(16, 16), incl=[[0.3, 0.3, 0.12], [0.63, 0.56, 0.13]], coh_law=2, coh=BL,
                     subscale=0, u_scale=1e-6, isv_scale=0.0, seed=6, open=(1e-7, 1.2e-2)),
    "coh_xn": dict(elem_type=0, n=(16, 16), incl=[[0.3, 0.3, 0.12], [0.63, 0.56, 0.13]], coh_law=3, coh=XN,
                   subscale=0, u_scale=1e-6, isv_scale=1.0, seed=7, open=(1e-6, 1e-3)),
    "coh_xnnu": dict(elem_type=0, n=(16, 16), incl=[[0.3, 0.3, 0.12], [0.63, 0.56, 0.13]], coh_law=4, coh=XN,
                     subscale=0, u_scale=1e-6, isv_scale=0.0, seed=8, open=(1e-6, 1e-3)),
    "coh_op": dict(elem_type=0, n=(16, 16), incl=[[0.3, 0.3, 0.12], [0.63, 0.56, 0.13]], coh_law=5, coh=OP,
                   subscale=0, u_scale=1e-6, isv_scale=1.0, seed=9, open=(1e-6, 1e-3)),
    "coh_opnu": dict(elem_type=0, n=(16, 16), incl=[[0.3, 0.3, 0.12], [0.63, 0.56, 0.13]], coh_law=6, coh=OP,
                     subscale=0, u_scale=1e-6, isv_scale=0.0, seed=10, open=(1e-6, 1e-3)),
    "coh_opaug": dict(elem_type=0, n=(16, 16), incl=[[0.3, 0.3, 0.12], [0.63, 0.56, 0.13]], coh_law=7, coh=OP,
                      subscale=0, u_scale=1e-6, isv_scale=1.0, seed=11, open=(1e-6, 1e-3)),
    "coh_opnuaug": dict(elem_type=0, n=(16, 16), incl=[[0.3, 0.3, 0.12], [0.63, 0.56, 0.13]], coh_law=8, coh=OP,
                        subscale=0, u_scale=1e-6, isv_scale=0.0, seed=12, open=(1e-6, 1e-3)),
    # trilinear and smoothed trilinear: openings across rise, plateau, fall and failure; the plain
    # laws read (never write) a committed maximum drawn over the same range, so points unload too
    "coh_tl": dict(elem_type=0, n=(16, 16), incl=[[0.3, 0.3, 0.12], [0.63, 0.56, 0.13]], coh_law=9, coh=TL,
                   subscale=0, u_scale=1e-6, isv_scale=6e-3, seed=28, open=(1e-7, 1.2e-2)),
    "coh_tlnu": dict(elem_type=0, n=(16, 16), incl=[[0.3, 0.3, 0.12], [0.63, 0.56, 0.13]], coh_law=10, coh=TL,
                     subscale=0, u_scale=1e-6, isv_scale=0.0, seed=29, open=(1e-7, 1.2e-2)),
    "coh_stl": dict(elem_type=0, n=(16, 16), incl=[[0.3, 0.3, 0.12], [0.63, 0.56, 0.13]], coh_law=11, coh=TL,
                    subscale=0, u_scale=1e-6, isv_scale=6e-3, seed=30, open=(1e-7, 1.2e-2)),
    "coh_stlnu": dict(elem_type=0, n=(16, 16), incl=[[0.3, 0.3, 0.12], [0.63, 0.56, 0.13]], coh_law=12, coh=TL,
                      subscale=0, u_scale=1e-6, isv_scale=0.0, seed=31, open=(1e-7, 1.2e-2)),
    # compression under a committed maximum: unloading points get the scaled penalty, loading points
    # with a maximum > 0 none (max_traction is only set on the unloading branch)
    "coh_stl_compression": dict(elem_type=0, n=(16, 16), incl=[[0.3, 0.3, 0.12], [0.63, 0.56, 0.13]], coh_law=11,
                                coh=TL, subscale=0, u_scale=1e-9, isv_scale=4e-8, seed=32, open=(-2e-8, -1e-9)),
    "coh_tlnu_compression": dict(elem_type=0, n=(16, 16), incl=[[0.3, 0.3, 0.12], [0.63, 0.56, 0.13]], coh_law=10,
                                 coh=TL, subscale=0, u_scale=1e-9, isv_scale=0.0, seed=33, open=(-2e-8, -1e-9)),
    "coh_bl_compression": dict(elem_type=0, n=(16, 16), incl=[[0.3, 0.3, 0.12], [0.63, 0.56, 0.13]], coh_law=1, coh=BL,
                               subscale=0, u_scale=1e-9, isv_scale=0.0, seed=14, open=(-2e-8, -1e-9)),
    "coh_opaug_compression": dict(elem_type=0, n=(16, 16), incl=[[0.3, 0.3, 0.12], [0.63, 0.56, 0.13]], coh_law=7, coh=OP,
                                  subscale=0, u_scale=1e-9, isv_scale=1.0, seed=15, open=(-4e-6, -1e-7)),
    "coh_opnuaug_compression": dict(elem_type=0, n=(16, 16), incl=[[0.3, 0.3, 0.12], [0.63, 0.56, 0.13]], coh_law=8, coh=OP,
                                    subscale=0, u_scale=1e-9, isv_scale=0.0, seed=16, open=(-4e-6, -1e-7)),
    "coh_bl_two_fibers_one_element": dict(elem_type=0, n=(8, 8), incl=[[0.3817, 0.5123, 0.1031], [0.6022, 0.4871, 0.1017]],
                                          coh_law=1, coh=BL, subscale=0, u_scale=1e-6, isv_scale=0.0, seed=13,
                                          open=(1e-7, 1.2e-2)),
    # two fibers 0.0076 apart: elements with a node in each fiber and one in the matrix are split
    # into two triangles and a Wachspress pentagon (4-point rule on each triangle of its fan)
    "lin_tri3_polygon": dict(elem_type=0, n=(8, 8), incl=[[0.5533, 0.6147, 0.1452], [0.8061, 0.5055, 0.0803]],
                             coh_law=0, coh=(0, 0, 0, 0), subscale=0, u_scale=1e-3, isv_scale=0.0, seed=17),
    "coh_bl_polygon": dict(elem_type=0, n=(8, 8), incl=[[0.5533, 0.6147, 0.1452], [0.8061, 0.5055, 0.0803]],
                           coh_law=1, coh=BL, subscale=0, u_scale=1e-6, isv_scale=0.0, seed=18, open=(1e-7, 1.2e-2)),
    # quad4 background elements: uncut rectangles with hx != hy (Dirichlet and periodic subscale
    # loading), and quad4 parents cut by fibers (Quad4::detection's polygonal cases: a triangle
    # and a pentagon, two quads, two fibers on one element with a quad between them), linear,
    # bilinear and Ortiz-Pandolfi interfaces, periodic with a macroscale strain
    "lin_quad4_uncut": dict(elem_type=1, n=(7, 5), incl=np.zeros((0, 3)), coh_law=0, coh=(0, 0, 0, 0), subscale=0,
                            u_scale=1e-3, isv_scale=0.0, seed=36),
    "lin_quad4_subscale": dict(elem_type=1, n=(9, 6), incl=np.zeros((0, 3)), coh_law=0, coh=(0, 0, 0, 0), subscale=1,
                               eps_macro=(0.01, -0.004, 0.002), u_scale=1e-3, isv_scale=0.0, seed=37),
    "lin_quad4_one_fiber": dict(elem_type=1, n=(8, 8), incl=[[0.5, 0.5, 0.23]], coh_law=0, coh=(0, 0, 0, 0),
                                subscale=0, u_scale=1e-3, isv_scale=0.0, seed=45),
    "lin_quad4_two_fibers_one_element": dict(elem_type=1, n=(8, 8), incl=[[0.5533, 0.6147, 0.1452], [0.8061, 0.5055, 0.0803]],
                                             coh_law=0, coh=(0, 0, 0, 0), subscale=0, u_scale=1e-3, isv_scale=0.0, seed=46),
    "lin_quad4_fiber_subscale": dict(elem_type=1, n=(9, 7), incl=[[0.47, 0.52, 0.21]], coh_law=0, coh=(0, 0, 0, 0),
                                     subscale=1, eps_macro=(0.01, -0.004, 0.002), u_scale=1e-3, isv_scale=0.0, seed=47),
    "coh_quad4_bl": dict(elem_type=1, n=(16, 16), incl=[[0.3, 0.3, 0.12], [0.63, 0.56, 0.13]], coh_law=1, coh=BL,
                         subscale=0, u_scale=1e-6, isv_scale=0.0, seed=48, open=(1e-7, 1.2e-2)),
    "coh_quad4_op": dict(elem_type=1, n=(16, 16), incl=[[0.3, 0.3, 0.12], [0.63, 0.56, 0.13]], coh_law=5, coh=OP,
                         subscale=0, u_scale=1e-6, isv_scale=1.0, seed=49, open=(1e-6, 1e-3)),
    "coh_quad4_bl_two_fibers_one_element": dict(elem_type=1, n=(8, 8), incl=[[0.5533, 0.6147, 0.1452], [0.8061, 0.5055, 0.0803]],
                                                coh_law=1, coh=BL, subscale=0, u_scale=1e-6, isv_scale=0.0, seed=50,
                                                open=(1e-7, 1.2e-2)),
    # transversely isotropic bounding plies: the element rows wholly above 0.8 / below 0.2 of the
    # height take the ply material (fiber axis x), with a fiber / sphere (linear and cohesive)
    # between them
    "lin_tri3_plies": dict(elem_type=0, n=(12, 10), incl=[[0.47, 0.52, 0.17]], coh_law=0, coh=(0, 0, 0, 0), subscale=0,
                           u_scale=1e-3, isv_scale=0.0, seed=38, ply_frac=0.2),
    "coh_bl_plies": dict(elem_type=0, n=(12, 10), incl=[[0.47, 0.52, 0.17]], coh_law=1, coh=BL, subscale=0,
                         u_scale=1e-6, isv_scale=0.0, seed=39, open=(1e-7, 1.2e-2), ply_frac=0.2),
    "lin_tet4_plies": dict(elem_type=2, n=(5, 5, 5), incl=[[0.52, 0.47, 0.49, 0.2]], coh_law=0, coh=(0, 0, 0, 0),
                           subscale=0, u_scale=1e-3, isv_scale=0.0, seed=40, ply_frac=0.2),
    # a fiber reaching into a ply: the matrix side of each cut ply element keeps the ply material
    "lin_tri3_ply_cut": dict(elem_type=0, n=(12, 10), incl=[[0.47, 0.26, 0.17], [0.66, 0.8, 0.11]], coh_law=0,
                             coh=(0, 0, 0, 0), subscale=0, u_scale=1e-3, isv_scale=0.0, seed=41, ply_frac=0.2,
                             ply_cut=1),
    "coh_bl_ply_cut": dict(elem_type=0, n=(12, 10), incl=[[0.47, 0.26, 0.17], [0.66, 0.8, 0.11]], coh_law=1, coh=BL,
                           subscale=0, u_scale=1e-6, isv_scale=0.0, seed=42, open=(1e-7, 1.2e-2), ply_frac=0.2,
                           ply_cut=1),
    "lin_tet4_ply_cut": dict(elem_type=2, n=(5, 5, 5), incl=[[0.52, 0.47, 0.49, 0.31]], coh_law=0, coh=(0, 0, 0, 0),
                             subscale=0, u_scale=1e-3, isv_scale=0.0, seed=43, ply_frac=0.2, ply_cut=1),
    "coh_tet4_bl_ply_cut": dict(elem_type=2, n=(5, 5, 5), incl=[[0.52, 0.47, 0.49, 0.31]], coh_law=1, coh=BL,
                                subscale=0, u_scale=1e-6, isv_scale=0.0, seed=44, open=(1e-7, 1.2e-2), ply_frac=0.2,
                                ply_cut=1),
    # tet4 (6 tets per hex): uncut, one sphere, periodic subscale with a macroscale strain, and
    # cohesive spheres (one node separated: tet + prism -> 4 tets and a CohTri3; two and two: two
    # prisms -> 6 tets and a CohQuad4)
    "lin_tet4_uncut": dict(elem_type=2, n=(4, 5, 3), incl=np.zeros((0, 4)), coh_law=0, coh=(0, 0, 0, 0), subscale=0,
                           u_scale=1e-3, isv_scale=0.0, seed=19),
    "lin_tet4_one_sphere": dict(elem_type=2, n=(5, 5, 5), incl=[[0.52, 0.47, 0.49, 0.31]], coh_law=0, coh=(0, 0, 0, 0),
                                subscale=0, u_scale=1e-3, isv_scale=0.0, seed=20),
    "lin_tet4_subscale": dict(elem_type=2, n=(5, 5, 5), incl=[[0.52, 0.47, 0.49, 0.31]], coh_law=0, coh=(0, 0, 0, 0),
                              subscale=1, eps_macro=(0.01, -0.004, 0.003, 0.002, -0.001, 0.0015), u_scale=1e-3,
                              isv_scale=0.0, seed=21),
    "coh_tet4_bl": dict(elem_type=2, n=(5, 5, 5), incl=[[0.52, 0.47, 0.49, 0.31]], coh_law=1, coh=BL, subscale=0,
                        u_scale=1e-6, isv_scale=0.0, seed=22, open=(1e-7, 1.2e-2)),
    "coh_tet4_xn": dict(elem_type=2, n=(5, 5, 5), incl=[[0.52, 0.47, 0.49, 0.31]], coh_law=3, coh=XN, subscale=0,
                        u_scale=1e-6, isv_scale=1.0, seed=23, open=(1e-6, 1e-3)),
    "coh_tet4_xnnu": dict(elem_type=2, n=(5, 5, 5), incl=[[0.52, 0.47, 0.49, 0.31]], coh_law=4, coh=XN, subscale=0,
                          u_scale=1e-6, isv_scale=0.0, seed=24, open=(1e-6, 1e-3)),
    "coh_tet4_op": dict(elem_type=2, n=(5, 5, 5), incl=[[0.52, 0.47, 0.49, 0.31]], coh_law=5, coh=OP, subscale=0,
                        u_scale=1e-6, isv_scale=1.0, seed=25, open=(1e-6, 1e-3)),
    "coh_tet4_opaug_two_spheres": dict(elem_type=2, n=(8, 7, 6), incl=[[0.3, 0.32, 0.35, 0.2], [0.7, 0.66, 0.62, 0.17]],
                                       coh_law=7, coh=OP, subscale=0, u_scale=1e-6, isv_scale=1.0, seed=26,
                                       open=(1e-6, 1e-3)),
    "coh_tet4_tl": dict(elem_type=2, n=(5, 5, 5), incl=[[0.52, 0.47, 0.49, 0.31]], coh_law=9, coh=TL, subscale=0,
                        u_scale=1e-6, isv_scale=6e-3, seed=34, open=(1e-7, 1.2e-2)),
    "coh_tet4_stlnu": dict(elem_type=2, n=(5, 5, 5), incl=[[0.52, 0.47, 0.49, 0.31]], coh_law=12, coh=TL, subscale=0,
                           u_scale=1e-6, isv_scale=0.0, seed=35, open=(1e-7, 1.2e-2)),
    "coh_tet4_bl_compression": dict(elem_type=2, n=(5, 5, 5), incl=[[0.52, 0.47, 0.49, 0.31]], coh_law=1, coh=BL,
                                    subscale=0, u_scale=1e-9, isv_scale=0.0, seed=27, open=(-2e-8, -1e-9)),
}


def case_arrays(c, n_free, n_const, n_isv):
    """Seeded DOF vector and committed internal variables of a bulk-only case."""
    rng = np.random.default_rng(c["seed"])
    U = rng.uniform(-c["u_scale"], c["u_scale"], n_free + n_const)
    isv = rng.uniform(0.0, c["isv_scale"], n_isv) if c["isv_scale"] > 0 else np.zeros(n_isv)
    return U, isv


def cohesive_state(c, node_dofs, n_free, n_const, elem_node_off, elem_nodes, elem_cut, elem_coh_off,
                   coh_struct, coh_struct_off, coh_qp_off, coh_R):
    """DOF vector of a cohesive case (see the module docstring).

    The topology arguments are the enriched-mesh tables (element node lists with enrichment nodes
    after the parent nodes, cohesive local node lists, per-qp rotation matrices whose last row is
    the interface normal)."""
    rng = np.random.default_rng(c["seed"])
    dim = 3 if c["elem_type"] == 2 else 2
    U = rng.uniform(-c["u_scale"], c["u_scale"], n_free + n_const)
    nd = node_dofs.reshape(-1, dim)
    lo, hi = c["open"]
    sign = 1.0 if lo > 0 else -1.0
    a, b = np.log(abs(lo)), np.log(abs(hi))
    for e in np.nonzero(elem_cut)[0]:
        nodes = elem_nodes[elem_node_off[e]:elem_node_off[e + 1]]
        for ce in range(elem_coh_off[e], elem_coh_off[e + 1]):
            cl = coh_struct[coh_struct_off[ce]:coh_struct_off[ce + 1]]
            nh = len(cl) // 2
            q0, q1 = coh_qp_off[ce], coh_qp_off[ce + 1]
            R = coh_R[q0 * dim * dim:q1 * dim * dim].reshape(-1, dim, dim).mean(axis=0)
            for k in range(nh):
                d_n = sign * np.exp(rng.uniform(min(a, b), max(a, b)))
                d_t = rng.uniform(-0.3, 0.3) * abs(d_n)
                jump = d_n * R[dim - 1] + d_t * R[0]
                U[nd[nodes[cl[k + nh]]]] = U[nd[nodes[cl[k]]]] + jump
    return U


def spec_kwargs(c):
    dim = 3 if c["elem_type"] == 2 else 2
    em = tuple(c.get("eps_macro", ())) + (0.0,) * (6 - len(c.get("eps_macro", ())))
    app = c["solve"][1] if "solve" in c else 0.01
    return dict(elem_type=c["elem_type"], n=c["n"], lo=(0.0,) * dim, hi=(1.0,) * dim,
                inclusions=np.array(c["incl"], dtype=np.float64), E_matrix=E_M, nu_matrix=NU_M, E_fiber=E_F,
                nu_fiber=NU_F, coh_law=c["coh_law"], coh=c["coh"], plane_strain=True, subscale=bool(c["subscale"]),
                eps_macro=em, app_strain=app, ply_frac=c.get("ply_frac", 0.0),
                ply=PLY if c.get("ply_frac", 0.0) > 0 else (0.0,) * 5)
