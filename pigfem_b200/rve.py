"""Seeded synthetic fiber-composite RVEs (the benchmark workloads).

The reference reads fiber layouts from CSV files (Tests/Main.cpp:744-860) and publishes no data
set; the workloads here are seeded synthetic layouts with the sizes and distributions of the
benchmark configurations:

* ``linear_2d``: unit square, 64 x 64 quads split into 8,192 tri3, ten fibers with radius
  ~ U[0.03, 0.06] and a minimum gap of 0.01, linear elastic, 1 % uniaxial strain prescribed on the
  right edge (Tests/Main.cpp:563-571): one K and R assembly.
* ``cohesive_2d``: unit square, N x N quads split into 2 N^2 tri3 (Mesh::generate_mesh), fibers
  placed by rejection sampling with radius ~ U[r_lo, r_hi], centre ~ U[r, 1-r]^2 and a minimum
  surface gap; bilinear cohesive law on every interface.
* ``linear_3d``: unit cube, N^3 hexes split into 6 tet4, spheres placed the same way, periodic
  subscale mode with unit macroscale strains.

Layouts are drawn from a counter-based Philox generator keyed by (workload, seed, request), so
the same key always gives the same RVE.  Layouts the reference cannot process are rejected:
a mesh node closer than 1e-9 r to a fiber surface (src/Mesh.cpp:2904-2911 stops the run), and in
3D any tet whose nodes see two different spheres (src/tet4.cpp:259-264).
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Optional

import numpy as np

from .capi import COH_BL, COH_NONE, TET4, TRI3, ProblemDesc

E_MATRIX, NU_MATRIX = 3.5e3, 0.35   # MPa
E_FIBER, NU_FIBER = 72e3, 0.22
# Bilinear interface: sigma_c = 50 MPa, delta_c2 = 5e-3 L, initial stiffness sigma_c / delta_c1
# with delta_c1 = delta_c2 / 1e4.
BL_PARAMS = (50.0, 5e-7, 5e-3, 0.0)


def philox(workload: int, seed: int, request: int = 0) -> np.random.Generator:
    """Counter-based stream keyed by (workload, seed); the request id sits in the second counter
    word, so each request owns 2^64 blocks before its stream could meet another's."""
    return np.random.Generator(np.random.Philox(key=np.array([workload, seed], dtype=np.uint64),
                                                counter=np.array([0, request, 0, 0], dtype=np.uint64)))


def place_fibers(rng: np.random.Generator, n_fibers: int, r_lo: float, r_hi: float, gap: float, dim: int,
                 max_attempts: int = 200000, radius_scale: float = 1.0, accept=None) -> np.ndarray:
    """Rejection sampling: returns an (n, dim+1) array of (centre, r); stops early if the
    attempt budget is spent (the achieved count is the array length).  `accept(c, r)` may veto a
    candidate."""
    out = []
    attempts = 0
    while len(out) < n_fibers and attempts < max_attempts:
        attempts += 1
        r = rng.uniform(r_lo, r_hi) * radius_scale
        c = rng.uniform(r, 1.0 - r, dim)
        ok = accept is None or accept(c, r)
        for f in out:
            if np.linalg.norm(c - f[:dim]) < r + f[dim] + gap:
                ok = False
                break
        if ok:
            out.append(np.concatenate([c, [r]]))
    return np.array(out).reshape(-1, dim + 1)


def sphere_box_ok(c: np.ndarray, r: float, n: int, tol_rel: float = 1e-12) -> bool:
    """The reference's sphere bounding box has upper z bound cy + r (src/InclusionSphere.cpp:158):
    grid nodes inside the sphere above that height are detected as outside, and the run stops on
    the first cut edge with no sign change.  Accept a sphere only if no grid node lies there."""
    zcut = c[1] + r
    if c[2] + r <= zcut:
        return True
    h = 1.0 / n
    lo = np.maximum(np.floor((c - r) / h).astype(int), 0)
    hi = np.minimum(np.ceil((c + r) / h).astype(int), n)
    k0 = max(lo[2], int(np.floor(zcut / h)))
    axes = [np.arange(lo[0], hi[0] + 1) * h, np.arange(lo[1], hi[1] + 1) * h, np.arange(k0, hi[2] + 1) * h]
    g = np.stack(np.meshgrid(*axes, indexing="ij"), -1).reshape(-1, 3)
    g = g[g[:, 2] > zcut]
    val = (((g - c) / r) ** 2).sum(1) - 1.0
    return not np.any(val <= tol_rel)


def surface_clearance_ok(fibers: np.ndarray, n: int, dim: int, tol_rel: float = 1e-9) -> bool:
    """No structured-grid node within tol_rel * r of any fiber surface."""
    h = 1.0 / n
    for f in fibers:
        c, r = f[:dim], f[dim]
        lo = np.maximum(np.floor((c - r) / h).astype(int) - 1, 0)
        hi = np.minimum(np.ceil((c + r) / h).astype(int) + 1, n)
        axes = [np.arange(lo[d], hi[d] + 1) * h for d in range(dim)]
        grid = np.stack(np.meshgrid(*axes, indexing="ij"), -1).reshape(-1, dim)
        d = np.sqrt(((grid - c) ** 2).sum(1))
        if np.any(np.abs(d - r) <= tol_rel * r):
            return False
    return True


@dataclass
class RVE:
    desc: ProblemDesc
    fibers: np.ndarray
    volume_fraction: float


def cohesive_2d(n: int = 512, n_fibers: int = 200, r_lo: float = 0.008, r_hi: float = 0.015, gap: float = 0.002,
                seed: int = 1, request: int = 0, workload: int = 1, app_strain: float = 0.02,
                coh_law: int = COH_BL, coh=BL_PARAMS, target_vf: Optional[float] = None) -> RVE:
    rng = philox(workload, seed, request)
    scale = 1.0
    if target_vf is not None:
        # radii scaled so the expected fiber area matches the target volume fraction
        mean_r2 = (r_hi ** 3 - r_lo ** 3) / (3 * (r_hi - r_lo))
        scale = math.sqrt(target_vf / (n_fibers * math.pi * mean_r2))
    for _ in range(20):
        fib = place_fibers(rng, n_fibers, r_lo, r_hi, gap, 2, radius_scale=scale)
        if surface_clearance_ok(fib, n, 2):
            break
    vf = float(np.sum(np.pi * fib[:, 2] ** 2))
    desc = ProblemDesc(elem_type=TRI3, n=(n, n), lo=(0.0, 0.0), hi=(1.0, 1.0), inclusions=fib,
                       E_matrix=E_MATRIX, nu_matrix=NU_MATRIX, E_fiber=E_FIBER, nu_fiber=NU_FIBER,
                       coh_law=coh_law, coh=coh, plane_strain=True, subscale=False, app_strain=app_strain)
    return RVE(desc, fib, vf)


def linear_2d(n: int = 64, n_fibers: int = 10, r_lo: float = 0.03, r_hi: float = 0.06, gap: float = 0.01,
              seed: int = 1, request: int = 0, workload: int = 0, app_strain: float = 0.01) -> RVE:
    """The 2D linear-elastic RVE: n x n quads split into tri3, seeded non-overlapping circular
    fibers, matrix / fiber isotropic linear elasticity (plane strain), no cohesive interfaces,
    u_x = app_strain * L on the right edge, u_x = 0 on the left, node 0 pinned."""
    return cohesive_2d(n=n, n_fibers=n_fibers, r_lo=r_lo, r_hi=r_hi, gap=gap, seed=seed, request=request,
                       workload=workload, app_strain=app_strain, coh_law=COH_NONE, coh=(0.0, 0.0, 0.0, 0.0))


def linear_3d(n: int = 64, n_spheres: int = 50, r_lo: float = 0.04, r_hi: float = 0.08, gap: float = 0.01,
              seed: int = 1, request: int = 0, workload: int = 3, max_redraws: int = 50) -> RVE:
    """Unit cube, n^3 hexes split into 6 tet4, seeded non-overlapping spheres, periodic subscale
    mode (node 0 pinned, macroscale strain) with eps_macro = e_1.  Spheres the reference's
    detection box would cut (sphere_box_ok) are redrawn; layouts with a mesh node on a sphere
    surface or a tet whose nodes see two different spheres are redrawn (the reference stops on
    both); the host set-up is the detection pre-check."""
    from .capi import PigfemError, Problem
    eps = (1.0, 0.0, 0.0, 0.0, 0.0, 0.0)
    for k in range(max_redraws):
        rng = philox(workload, seed, request * 1000 + k)
        fib = place_fibers(rng, n_spheres, r_lo, r_hi, gap, 3, accept=lambda c, r: sphere_box_ok(c, r, n))
        if not surface_clearance_ok(fib, n, 3):
            continue
        desc = ProblemDesc(elem_type=TET4, n=(n, n, n), lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), inclusions=fib,
                           E_matrix=E_MATRIX, nu_matrix=NU_MATRIX, E_fiber=E_FIBER, nu_fiber=NU_FIBER,
                           plane_strain=False, subscale=True, eps_macro=eps)
        try:
            Problem(desc, device=False).close()
        except PigfemError as e:
            if e.code in (3, 4):
                continue
            raise
        vf = float(np.sum(4.0 / 3.0 * np.pi * fib[:, 3] ** 3))
        return RVE(desc, fib, vf)
    raise RuntimeError("no admissible sphere layout found")


def cohesive_batch(count: int = 256, seed: int = 1, n_lo: int = 32, n_hi: int = 256, fib_lo: int = 5,
                   fib_hi: int = 120, vf_lo: float = 0.2, vf_hi: float = 0.5, gap: float = 0.002,
                   workload: int = 4, max_attempts: int = 20000):
    """Independent 2D cohesive RVEs of uneven size: grid side N ~ log-uniform[n_lo, n_hi], fiber
    count ~ U{fib_lo..fib_hi}, radii U[0.8, 1.2] x the mean radius of a volume fraction drawn from
    U[vf_lo, vf_hi]; rejection sampling with capped attempts (the achieved volume fraction is
    recorded); bilinear cohesive interfaces as in cohesive_2d.  RVE k is keyed by request k."""
    out = []
    for k in range(count):
        rng = philox(workload, seed, k)
        n = int(round(math.exp(rng.uniform(math.log(n_lo), math.log(n_hi)))))
        nf = int(rng.integers(fib_lo, fib_hi + 1))
        vf = float(rng.uniform(vf_lo, vf_hi))
        r_mean = math.sqrt(vf / (nf * math.pi))
        for _ in range(20):
            fib = place_fibers(rng, nf, 0.8 * r_mean, 1.2 * r_mean, gap, 2, max_attempts=max_attempts)
            if len(fib) and surface_clearance_ok(fib, n, 2):
                break
        vf_got = float(np.sum(np.pi * fib[:, 2] ** 2))
        desc = ProblemDesc(elem_type=TRI3, n=(n, n), lo=(0.0, 0.0), hi=(1.0, 1.0), inclusions=fib,
                           E_matrix=E_MATRIX, nu_matrix=NU_MATRIX, E_fiber=E_FIBER, nu_fiber=NU_FIBER,
                           coh_law=COH_BL, coh=BL_PARAMS, plane_strain=True, subscale=False, app_strain=0.02)
        out.append(RVE(desc, fib, vf_got))
    return out


def interface_state(problem, seed: int = 0, open_lo: float = 1e-7, open_hi: float = 6e-3, u_scale: float = 1e-6):
    """A displacement field (node-major) with seeded tensile openings at every cohesive interface
    of `problem` (a :class:`capi.Problem`): :func:`interface_state_tables` on its set-up tables."""
    return interface_state_tables(
        problem.dim, problem.n_nodes, problem.debug("cut_node_off"), problem.debug("cut_nodes"),
        problem.debug("cut_coh_off"), problem.debug("coh_local_off"), problem.debug("coh_local"),
        problem.debug("coh_qp_off"), problem.debug("cqp_R"), seed=seed, open_lo=open_lo, open_hi=open_hi,
        u_scale=u_scale)


def interface_state_tables(dim: int, n_nodes: int, cut_node_off, cut_nodes, cut_coh_off, coh_local_off, coh_local,
                           coh_qp_off, cqp_R, seed: int = 0, open_lo: float = 1e-7, open_hi: float = 6e-3,
                           u_scale: float = 1e-6):
    """A displacement field (node-major) with seeded tensile openings at every cohesive interface:
    each '+' enrichment node is displaced from its '-' partner along the mean normal of the
    cohesive elements that hold the pair, by a log-uniform opening in [open_lo, open_hi] plus a
    tangential slip of up to 0.3 of it, so the bilinear law runs through its loading, softening
    and failed branches while every cohesive point stays in tension.  Bulk displacements are small
    random values.

    The tables describe the enriched mesh in the reference's own terms, so the same state can be
    built from this library's set-up or from the reference's mesh: the cut elements' node lists
    (parent nodes, then enrichment nodes; node ids standard first, then enrichment), the range of
    cohesive elements of each cut element, each cohesive element's local node list ('-' half, then
    '+' half, indices into its cut element's node list), and the rotation of every cohesive
    quadrature point (dim x dim, last row the normal)."""
    cut_node_off, cut_nodes, cut_coh_off = (np.asarray(a) for a in (cut_node_off, cut_nodes, cut_coh_off))
    coh_local_off, coh_local, coh_qp_off = (np.asarray(a) for a in (coh_local_off, coh_local, coh_qp_off))
    rng = np.random.default_rng(seed)
    U = rng.uniform(-u_scale, u_scale, n_nodes * dim).reshape(-1, dim)
    n_ce = len(coh_local_off) - 1
    if n_ce <= 0:
        return np.ascontiguousarray(U.reshape(-1))
    R = np.asarray(cqp_R, dtype=np.float64).reshape(-1, dim, dim)
    ce_cut = np.repeat(np.arange(len(cut_coh_off) - 1), np.diff(cut_coh_off))
    Rm = np.add.reduceat(R, coh_qp_off[:-1], axis=0) / np.diff(coh_qp_off)[:, None, None]
    nh = np.diff(coh_local_off) // 2
    # every ('-', '+') node pair of every cohesive element
    pair_ce = np.repeat(np.arange(n_ce), nh)
    pair_k = np.arange(len(pair_ce)) - np.repeat(np.cumsum(nh) - nh, nh)
    base = coh_local_off[pair_ce]
    first = cut_node_off[ce_cut[pair_ce]]
    minus = cut_nodes[first + coh_local[base + pair_k]]
    plus = cut_nodes[first + coh_local[base + pair_k + nh[pair_ce]]]
    # mean normal and tangent of each '+' node over the cohesive elements holding it
    nsum = np.zeros((n_nodes, dim))
    tsum = np.zeros((n_nodes, dim))
    np.add.at(nsum, plus, Rm[pair_ce, dim - 1])
    np.add.at(tsum, plus, Rm[pair_ce, 0])
    nodes_p, idx = np.unique(plus, return_index=True)
    nodes_m = minus[idx]
    nrm = nsum[nodes_p] / np.linalg.norm(nsum[nodes_p], axis=1)[:, None]
    tng = tsum[nodes_p] / np.maximum(np.linalg.norm(tsum[nodes_p], axis=1), 1e-300)[:, None]
    a, b = math.log(open_lo), math.log(open_hi)
    draws = rng.uniform(0.0, 1.0, (len(nodes_p), 2))
    dn = np.exp(a + (b - a) * draws[:, 0])
    dt = (-0.3 + 0.6 * draws[:, 1]) * dn
    U[nodes_p] = U[nodes_m] + dn[:, None] * nrm + dt[:, None] * tng
    return np.ascontiguousarray(U.reshape(-1))
