// pg_kernels.cuh -- the assembly kernels.
//
//   k_coh_elements   one lane per cohesive quadrature point, the lanes of an element together:
//                    opening delta = R sum_n N_n (U+ - U-), the traction-separation law with its
//                    internal-variable update and damage zone, and the element's cohesive blocks
//                    and tractions (src/Utilities.cpp:528-594).  FP64.
//   k_cut_volumetric run once at set-up: the cut elements' volumetric (linear, state-independent)
//                    element matrices from sub-element quadrature with enriched B-matrices
//                    (src/Assembler.cpp:223-274), cached for every later assembly.  FP64.
//   k_rows_general   one lane group per DOF node (row owner) for every node the structured stencil
//                    path (pg_stencil.cuh) does not take: boundary rows, nodes of cut elements and
//                    enrichment nodes; uncut elements are recomputed from node coordinates; for cut
//                    elements the cached volumetric block row is combined with the nodal
//                    displacements and the cohesive elements' blocks (src/Assembler.cpp:278-365).
//                    Every CSR value is written once.
// No atomics anywhere: every row has one owner and sums in a fixed order, so results are
// bit-reproducible from run to run.
#pragma once

#include "pg_device.cuh"

namespace pgd {

// Geometry of an affine simplex (tri3 / tet4): physical gradients g[n][d] and the Jacobian
// determinant.  Jac(a,i) = sum_n dN_n/dr_a x_n[i] (Elem::transform_gradients), i.e. x_{a+1} - x_0;
// inverse = adjugate * (1/det) (Utilities::inverse).
template <int DIM, typename T>
__device__ __forceinline__ void simplex_geom(const T (*x)[DIM], T (*g)[DIM], T* J) {
  if (DIM == 2) {
    const T j00 = x[1][0] - x[0][0], j01 = x[1][1] - x[0][1];
    const T j10 = x[2][0] - x[0][0], j11 = x[2][1] - x[0][1];
    const T det = j00 * j11 - j01 * j10;
    const T s = T(1) / det;
    const T i00 = j11 * s, i11 = j00 * s, i01 = (T(-1) * j01) * s, i10 = (T(-1) * j10) * s;
    g[0][0] = -(i00 + i01); g[0][1] = -(i10 + i11);
    g[1][0] = i00; g[1][1] = i10;
    g[2][0] = i01; g[2][1] = i11;
    *J = det;
  } else {
    T a[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int i = 0; i < 3; ++i) a[r][i] = x[r + 1][i] - x[0][i];
    const T det = a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) - a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]) +
                  a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
    T R[3][3];
    R[0][0] = a[1][1] * a[2][2] - a[2][1] * a[1][2];
    R[0][1] = T(-1) * (a[0][1] * a[2][2] - a[2][1] * a[0][2]);
    R[0][2] = a[0][1] * a[1][2] - a[1][1] * a[0][2];
    R[1][0] = T(-1) * (a[1][0] * a[2][2] - a[2][0] * a[1][2]);
    R[1][1] = a[0][0] * a[2][2] - a[2][0] * a[0][2];
    R[1][2] = T(-1) * (a[0][0] * a[1][2] - a[1][0] * a[0][2]);
    R[2][0] = a[1][0] * a[2][1] - a[2][0] * a[1][1];
    R[2][1] = T(-1) * (a[0][0] * a[2][1] - a[2][0] * a[0][1]);
    R[2][2] = a[0][0] * a[1][1] - a[1][0] * a[0][1];
    const T s = T(1) / det;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      g[1][i] = R[i][0] * s; g[2][i] = R[i][1] * s; g[3][i] = R[i][2] * s;
      g[0][i] = -(g[1][i] + g[2][i] + g[3][i]);
    }
    *J = det;
  }
}

// sigma = D eps with the linear-elastic zero pattern (LinearElasticIsotropicMaterial::computeStress)
template <int DIM, typename T>
__device__ __forceinline__ void lei_stress(const T* D, const T* e, T* s) {
  if (DIM == 2) {
    s[0] = D[0] * e[0] + D[1] * e[1];
    s[1] = D[3] * e[0] + D[4] * e[1];
    s[2] = D[8] * e[2];
  } else {
    s[0] = D[0] * e[0] + D[1] * e[1] + D[2] * e[2];
    s[1] = D[6] * e[0] + D[7] * e[1] + D[8] * e[2];
    s[2] = D[12] * e[0] + D[13] * e[1] + D[14] * e[2];
    s[3] = D[21] * e[3];
    s[4] = D[28] * e[4];
    s[5] = D[35] * e[5];
  }
}

// Row q of B_a^T D for node gradient ga ("part" of the reference's SmallStrainKFast).
template <int DIM, typename T>
__device__ __forceinline__ void bt_d_row(const T* D, const T* ga, int q, T* part) {
  if (DIM == 2) {
    if (q == 0) { part[0] = ga[0] * D[0] + ga[1] * D[6]; part[1] = ga[0] * D[1] + ga[1] * D[7]; part[2] = ga[0] * D[2] + ga[1] * D[8]; }
    else        { part[0] = ga[1] * D[3] + ga[0] * D[6]; part[1] = ga[1] * D[4] + ga[0] * D[7]; part[2] = ga[1] * D[5] + ga[0] * D[8]; }
  } else {
#pragma unroll
    for (int v = 0; v < 6; ++v) {
      if (q == 0) part[v] = ga[0] * D[0 * 6 + v] + ga[2] * D[4 * 6 + v] + ga[1] * D[5 * 6 + v];
      else if (q == 1) part[v] = ga[1] * D[1 * 6 + v] + ga[2] * D[3 * 6 + v] + ga[0] * D[5 * 6 + v];
      else part[v] = ga[2] * D[2 * 6 + v] + ga[1] * D[3 * 6 + v] + ga[0] * D[4 * 6 + v];
    }
  }
}
// (part . B_b)(:, q2)
template <int DIM, typename T>
__device__ __forceinline__ T part_b(const T* part, const T* gb, int q2) {
  if (DIM == 2) return (q2 == 0) ? part[0] * gb[0] + part[2] * gb[1] : part[1] * gb[1] + part[2] * gb[0];
  if (q2 == 0) return part[0] * gb[0] + part[4] * gb[2] + part[5] * gb[1];
  if (q2 == 1) return part[1] * gb[1] + part[3] * gb[2] + part[5] * gb[0];
  return part[2] * gb[2] + part[3] * gb[1] + part[4] * gb[0];
}
// (B_a^T sigma)[q]
template <int DIM, typename T>
__device__ __forceinline__ T bt_sig(const T* ga, const T* s, int q) {
  if (DIM == 2) return (q == 0) ? ga[0] * s[0] + ga[1] * s[2] : ga[1] * s[1] + ga[0] * s[2];
  if (q == 0) return ga[0] * s[0] + ga[2] * s[4] + ga[1] * s[5];
  if (q == 1) return ga[1] * s[1] + ga[2] * s[3] + ga[0] * s[5];
  return ga[2] * s[2] + ga[1] * s[3] + ga[0] * s[4];
}
// Voigt strain of a set of nodes
template <int DIM, typename T>
__device__ __forceinline__ void add_strain(const T* g, const T* u, T* e) {
  if (DIM == 2) {
    e[0] += g[0] * u[0]; e[1] += g[1] * u[1]; e[2] += g[1] * u[0] + g[0] * u[1];
  } else {
    e[0] += g[0] * u[0]; e[1] += g[1] * u[1]; e[2] += g[2] * u[2];
    e[3] += g[2] * u[1] + g[1] * u[2];
    e[4] += g[2] * u[0] + g[0] * u[2];
    e[5] += g[1] * u[0] + g[0] * u[1];
  }
}

// Weight sum of the reference rules for the uncut parents: tri3 order 3 and tet4 order 3.
__device__ __host__ inline double tri4_wsum() { return ((-0.28125 + 0.260416666666666666666666666666665) + 0.260416666666666666666666666666665) + 0.260416666666666666666666666666665; }
__device__ __host__ inline double tet5_wsum() { return (((-0.8 + 0.45) + 0.45) + 0.45) + 0.45; }

// Block (la, lb) of an uncut simplex with the given nodes: kb = w (B_la^T D B_lb) (WANT_K); with
// want_r also the residual of row la, rv = w (B_la^T sigma).  Geometry from the node coordinates,
// stress from U (+ eps_macro).
template <int DIM, bool WANT_K = true>
__device__ __forceinline__ void simplex_block(const DevProblem& P, int4 nodes, int la, int lb, const double* D,
                                              double (*kb)[DIM], double* rv, bool want_r) {
  constexpr int NPE = DIM + 1;
  constexpr int NV = (DIM == 2) ? 3 : 6;
  const int nd[4] = {nodes.x, nodes.y, nodes.z, nodes.w};
  double x[NPE][DIM], g[NPE][DIM], J;
#pragma unroll
  for (int n = 0; n < NPE; ++n) load_node<DIM>(P.X, nd[n], x[n]);
  simplex_geom<DIM, double>(x, g, &J);
  const double wgt = J * ((DIM == 2) ? tri4_wsum() : tet5_wsum());
  double ga[DIM], gb[DIM];
#pragma unroll
  for (int d = 0; d < DIM; ++d) { ga[d] = g[0][d]; gb[d] = g[0][d]; }
#pragma unroll
  for (int n = 1; n < NPE; ++n) {
    if (la == n)
#pragma unroll
      for (int d = 0; d < DIM; ++d) ga[d] = g[n][d];
    if (lb == n)
#pragma unroll
      for (int d = 0; d < DIM; ++d) gb[d] = g[n][d];
  }
  if constexpr (WANT_K) {
#pragma unroll
    for (int q = 0; q < DIM; ++q) {
      double part[NV];
      bt_d_row<DIM, double>(D, ga, q, part);
#pragma unroll
      for (int q2 = 0; q2 < DIM; ++q2) kb[q][q2] = wgt * part_b<DIM, double>(part, gb, q2);
    }
  }
  if (want_r) {
    double eps[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) eps[v] = 0.0;
#pragma unroll
    for (int n = 0; n < NPE; ++n) {
      double u[DIM];
      load_node<DIM>(P.U, nd[n], u);
      add_strain<DIM, double>(g[n], u, eps);
    }
    if (P.subscale) {
#pragma unroll
      for (int v = 0; v < NV; ++v) eps[v] += P.eps_macro[v];
    }
    double sig[NV];
    lei_stress<DIM, double>(D, eps, sig);
#pragma unroll
    for (int q = 0; q < DIM; ++q) rv[q] = wgt * bt_sig<DIM, double>(ga, sig, q);
  }
}

// Shared memory of one lane group of general_rows: slab_slots blocks of DIM x DIM, the node's
// residual (4 doubles reserved), the per-slot residual partials of the static part
// (slab_slots x DIM), then one scratch record per lane (general_lane_doubles).
__host__ __device__ constexpr int general_lane_doubles(int dim, int npe) { return npe * dim * dim + dim + 2; }
__host__ __device__ inline int general_scratch_offset(int slab_slots, int dim) {
  return (slab_slots * dim * dim + 4 + slab_slots * dim + 1) & ~1;   // even: 16-byte aligned
}
__host__ __device__ inline int general_slab_doubles(int slab_slots, int dim, int lanes, int npe = 0) {
  // even (16-byte aligned groups) and 2 mod 4, so consecutive groups start on different banks
  if (npe == 0) npe = dim + 1;
  int n = (general_scratch_offset(slab_slots, dim) + lanes * general_lane_doubles(dim, npe) + 1) & ~1;
  return (n % 4 == 0) ? n + 2 : n;
}

// slab block += v (DIM x DIM); 16-byte shared-memory accesses in 2D
template <int DIM>
__device__ __forceinline__ void slab_add(double* ak, const double* v) {
  if constexpr (DIM == 2) {
    double2* a2 = reinterpret_cast<double2*>(ak);
    double2 t0 = a2[0], t1 = a2[1];
    t0.x += v[0]; t0.y += v[1]; t1.x += v[2]; t1.y += v[3];
    a2[0] = t0; a2[1] = t1;
  } else {
#pragma unroll
    for (int i = 0; i < DIM * DIM; ++i) ak[i] += v[i];
  }
}

// Point qp of the quad4 2 x 2 Gauss rule (src/quad4.cpp:108-127: the edge points -+1/sqrt(3),
// qp -> (qp % 2, qp / 2), weights 1 x 1) on the bilinear map of the nodes x: the physical
// gradients g of the four shape functions (Jacobian J(a, i) = sum_k dN_k/dr_a x_k[i], its
// inverse by the adjugate, Elem::transform_gradients, src/elem.cpp:115-139) and the weight J W.
__device__ __forceinline__ void quad4_point(const double (*x)[2], int qp, double (*g)[2], double* w) {
  const double kG = 0.57735026918962576450914878050196;
  const double r = (qp % 2) ? kG : -kG, s = (qp / 2) ? kG : -kG;
  const double dN[4][2] = {{-0.25 * (1.0 - s), -0.25 * (1.0 - r)}, {0.25 * (1.0 - s), -0.25 * (1.0 + r)},
                           {0.25 * (1.0 + s), 0.25 * (1.0 + r)}, {-0.25 * (1.0 + s), 0.25 * (1.0 - r)}};
  double J[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int k = 0; k < 4; ++k) J[a][i] += dN[k][a] * x[k][i];
  const double det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
  const double sc = 1.0 / det;
  const double R[2][2] = {{J[1][1] * sc, (-1.0 * J[0][1]) * sc}, {(-1.0 * J[1][0]) * sc, J[0][0] * sc}};
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int i = 0; i < 2; ++i) g[k][i] = R[i][0] * dN[k][0] + R[i][1] * dN[k][1];
  *w = det * (1.0 * 1.0);
}

// Block row la of an uncut element with the given nodes: blk[b] = sum over its points of
// w (B_la^T D B_b) for every element node b (NPE blocks of DIM x DIM, row-major), and its
// residual rv = sum w (B_la^T sigma).  Simplices (NPE = DIM + 1) have constant gradients, so
// their order-3 points are summed into one weight (the products of simplex_block); quad4
// (DIM = 2, NPE = 4) sums its four Gauss points.  Geometry from the node coordinates, stress
// from U (+ eps_macro).
template <int DIM, int NPE = DIM + 1>
__device__ __forceinline__ void uncut_block_row(const DevProblem& P, int4 nodes, int la, const double* D, double* blk,
                                                double* rv) {
  constexpr int NV = (DIM == 2) ? 3 : 6;
  constexpr int D2 = DIM * DIM;
  const int nd[4] = {nodes.x, nodes.y, nodes.z, nodes.w};
  if constexpr (DIM == 2 && NPE == 4) {
    double x[4][2], u[4][2];
#pragma unroll
    for (int n = 0; n < 4; ++n) { load_node<2>(P.X, nd[n], x[n]); load_node<2>(P.U, nd[n], u[n]); }
    double kb[4][4], r[2] = {0.0, 0.0};
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
      for (int i = 0; i < 4; ++i) kb[b][i] = 0.0;
#pragma unroll
    for (int qp = 0; qp < 4; ++qp) {
      double g[4][2], w;
      quad4_point(x, qp, g, &w);
      double ga[2] = {g[0][0], g[0][1]};
#pragma unroll
      for (int n = 1; n < 4; ++n)
        if (la == n) { ga[0] = g[n][0]; ga[1] = g[n][1]; }
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        double part[3];
        bt_d_row<2, double>(D, ga, q, part);
#pragma unroll
        for (int b = 0; b < 4; ++b)
#pragma unroll
          for (int q2 = 0; q2 < 2; ++q2) kb[b][q * 2 + q2] += w * part_b<2, double>(part, g[b], q2);
      }
      double eps[3] = {0.0, 0.0, 0.0};
#pragma unroll
      for (int n = 0; n < 4; ++n) add_strain<2, double>(g[n], u[n], eps);
      if (P.subscale) {
#pragma unroll
        for (int v = 0; v < 3; ++v) eps[v] += P.eps_macro[v];
      }
      double sig[3];
      lei_stress<2, double>(D, eps, sig);
#pragma unroll
      for (int q = 0; q < 2; ++q) r[q] += w * bt_sig<2, double>(ga, sig, q);
    }
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
      for (int i = 0; i < 4; ++i) blk[b * D2 + i] = kb[b][i];
    rv[0] = r[0];
    rv[1] = r[1];
  } else {
    double x[NPE][DIM], g[NPE][DIM], J;
#pragma unroll
    for (int n = 0; n < NPE; ++n) load_node<DIM>(P.X, nd[n], x[n]);
    simplex_geom<DIM, double>(x, g, &J);
    const double wgt = J * ((DIM == 2) ? tri4_wsum() : tet5_wsum());
    double ga[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) ga[d] = g[0][d];
#pragma unroll
    for (int n = 1; n < NPE; ++n)
      if (la == n)
#pragma unroll
        for (int d = 0; d < DIM; ++d) ga[d] = g[n][d];
#pragma unroll
    for (int q = 0; q < DIM; ++q) {
      double part[NV];
      bt_d_row<DIM, double>(D, ga, q, part);
#pragma unroll
      for (int b = 0; b < NPE; ++b)
#pragma unroll
        for (int q2 = 0; q2 < DIM; ++q2) blk[b * D2 + q * DIM + q2] = wgt * part_b<DIM, double>(part, g[b], q2);
    }
    double eps[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) eps[v] = 0.0;
#pragma unroll
    for (int n = 0; n < NPE; ++n) {
      double u[DIM];
      load_node<DIM>(P.U, nd[n], u);
      add_strain<DIM, double>(g[n], u, eps);
    }
    if (P.subscale) {
#pragma unroll
      for (int v = 0; v < NV; ++v) eps[v] += P.eps_macro[v];
    }
    double sig[NV];
    lei_stress<DIM, double>(D, eps, sig);
#pragma unroll
    for (int q = 0; q < DIM; ++q) rv[q] = wgt * bt_sig<DIM, double>(ga, sig, q);
  }
}

// Static residual of a general node next to cut elements: sum over its neighbour slots (in slot
// order) of the static block times the slot node's displacement, then the macroscale-strain
// response.  `part` holds the per-slot products (slot-major, DIM each), written by the caller's
// lanes; the sum runs on one lane, so it does not depend on how many lanes formed the products.
template <int DIM>
__device__ __forceinline__ void static_resid_sum(const DevProblem& P, int node, int nn, const double* part,
                                                 const double* eps, double* r) {
  constexpr int NV = (DIM == 2) ? 3 : 6;
#pragma unroll
  for (int q = 0; q < DIM; ++q) r[q] = 0.0;
  for (int k = 0; k < nn; ++k)
#pragma unroll
    for (int q = 0; q < DIM; ++q) r[q] += part[k * DIM + q];
  if (P.subscale) {
    const double* Gs = P.stat_g + (size_t)node * DIM * NV;
#pragma unroll
    for (int q = 0; q < DIM; ++q)
#pragma unroll
      for (int v = 0; v < NV; ++v) r[q] += __ldg(&Gs[q * NV + v]) * eps[v];
  }
}

// Product of static slot k of a general node with the slot node's displacement (one slot's
// contribution to the static residual).
template <int DIM>
__device__ __forceinline__ void static_slot_product(const DevProblem& P, int s0, int k, double* out) {
  constexpr int D2 = DIM * DIM;
  const double* S = P.stat + (size_t)(s0 + k) * D2;
  double u[DIM];
  load_node<DIM>(P.U, __ldg(&P.stat_node[s0 + k]), u);
#pragma unroll
  for (int q = 0; q < DIM; ++q) {
    double v = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) v += __ldg(&S[q * DIM + d]) * u[d];
    out[q] = v;
  }
}

// The cohesive element's block (n1, n2) and the traction at n1 for a row node at cohesive place
// cpa = (element << 5 | n1): sgn * B_{n1 % nh, n2 % nh} and sgn * t_{n1 % nh}
// (cohesiveKFast / cohesiveInternalForceFast signs).
template <int DIM>
__device__ __forceinline__ void coh_block_add(const DevProblem& P, int cpa, int cpb, double* blk) {
  constexpr int D2 = DIM * DIM;
  const int ce = cpa >> 5, n1 = cpa & 31, n2 = cpb & 31;
  const int nh = __ldg(&P.coh_nh[ce]);
  const double sgn = ((n1 >= nh) == (n2 >= nh)) ? 1.0 : -1.0;
  const double* B = P.kcoh + __ldg(&P.kc_off[ce]) + ((n1 % nh) * nh + (n2 % nh)) * D2;
#pragma unroll
  for (int i = 0; i < D2; ++i) blk[i] = sgn * B[i];
}
template <int DIM>
__device__ __forceinline__ void coh_traction(const DevProblem& P, int cpa, double* t) {
  constexpr int D2 = DIM * DIM;
  const int ce = cpa >> 5, n1 = cpa & 31;
  const int nh = __ldg(&P.coh_nh[ce]);
  const double sgn = (n1 >= nh) ? 1.0 : -1.0;
  const double* tp = P.kcoh + __ldg(&P.kc_off[ce]) + nh * nh * D2 + (n1 % nh) * DIM;
#pragma unroll
  for (int q = 0; q < DIM; ++q) t[q] = sgn * tp[q];
}

// Row assembly for the DOF nodes the stencil path does not take (boundary rows, nodes of cut
// elements, enrichment nodes): one lane group of L threads per DOF node, its rows in a
// shared-memory slab.  The slab starts from the node's static part (the cut elements' volumetric
// blocks summed per neighbour slot at set-up; zero for nodes without cut elements) and the
// residual from the static blocks times the displacements plus the macroscale-strain response.
// The node's adjacent elements then follow in adjacency order (cut elements first):
//   * a cut element the row node is on a cohesive element of adds that cohesive element's blocks
//     and traction (k_coh_elements left them in kcoh), its lanes taking the element's nodes;
//   * the uncut elements are taken L at a time: lane k recomputes element e0 + k from the node
//     coordinates and writes its whole block row and residual to its scratch record, then the
//     lanes add the records into the slab in entry order, each lane owning the slots s = k,
//     k + L, ... (an element's nodes have distinct slots), and lane 0 adds the residuals.
// Every sum therefore runs in a fixed order that does not depend on L.  Finally the group writes
// every CSR value of the node's rows exactly once.
//   gdesc[node]      int4 {adjacency begin, adjacency count, neighbour begin, neighbour count}
//   growd[node]      3*DIM ints: global DOF of each row, first slot in the row's F block, in its C block
//   adesc[entry]     int4 {element, local node | nodes of a cut element << 8, slots (uncut: 8 bits per
//                    node; cut: offset into adj_slots), material (uncut)}
//   aresd[entry]     int4: uncut {element nodes (-1 padded)}; cut {cut element, its first node in
//                    cut_nodes, the row node's cohesive place (element << 5 | position) or -1, 0}
//   nbr_pre[slot]    free DOFs of the node's neighbours before this one (row positions)
// `valid` is uniform over the group, and the group synchronises only its own lanes.  `slab` is the
// group's general_slab_doubles(slab_slots, DIM, L) doubles.  (Residual-only assemblies use
// k_rows_general_resid.)
template <int DIM, int L, int NPE = DIM + 1>
__device__ __forceinline__ void general_rows(const DevProblem& P, int node, bool valid, double* slab, int slab_slots) {
  constexpr int D2 = DIM * DIM;
  constexpr int LD = general_lane_doubles(DIM, NPE);
  if (!valid) return;
  const int g = threadIdx.x % L;
  const unsigned gmask = (L >= 32) ? 0xffffffffu : (((1u << L) - 1u) << ((threadIdx.x & 31) / L * L));
  const int4 gd = __ldg(&P.gdesc[node]);
  const int nn = gd.w;
  const bool stat = node < P.n_stat;
  double* rs = slab + nn * D2;             // residual of the node's rows
  double* part = rs + 4;                   // per-slot residual partials of the static part
  double* scr = slab + general_scratch_offset(slab_slots, DIM);
  if (stat) {
    const int s0 = __ldg(&P.stat_slot_off[node]);
    const double* S = P.stat + (size_t)s0 * D2;
    for (int i = g; i < nn * D2; i += L) slab[i] = __ldg(&S[i]);
    for (int k = g; k < nn; k += L) static_slot_product<DIM>(P, s0, k, part + k * DIM);
  } else {
    for (int i = g; i < nn * D2; i += L) slab[i] = 0.0;
  }
  __syncwarp(gmask);
  if (g == 0) {
    double r[DIM];
    if (stat) static_resid_sum<DIM>(P, node, nn, part, P.eps_macro, r);
    else
#pragma unroll
      for (int q = 0; q < DIM; ++q) r[q] = 0.0;
#pragma unroll
    for (int q = 0; q < DIM; ++q) rs[q] = r[q];
  }
  __syncwarp(gmask);
  // cut entries (first in the adjacency order): the cohesive element the row node is on
  int e = 0;
  for (; e < gd.y; ++e) {
    const int4 ad = __ldg(&P.adesc[gd.x + e]);
    const int mn = ad.y >> 8;
    if (mn == 0) break;
    const int4 ax = __ldg(&P.aresd[gd.x + e]);
    const int cpa = ax.z;
    if (cpa < 0) continue;
    for (int b = g; b < mn; b += L) {
      const int cpb = __ldg(&P.cohpos[ax.y + b]);
      if (cpb >= 0 && (cpb >> 5) == (cpa >> 5)) {
        double blk[D2];
        coh_block_add<DIM>(P, cpa, cpb, blk);
        slab_add<DIM>(slab + __ldg(&P.adj_slots[ad.z + b]) * D2, blk);
      }
    }
    if (g == 0) {
      double t[DIM];
      coh_traction<DIM>(P, cpa, t);
#pragma unroll
      for (int q = 0; q < DIM; ++q) rs[q] += t[q];
    }
    __syncwarp(gmask);
  }
  // uncut entries, L at a time
  for (int e0 = e; e0 < gd.y; e0 += L) {
    double* my = scr + g * LD;
    unsigned z = 0u;
    if (e0 + g < gd.y) {
      const int4 ad = __ldg(&P.adesc[gd.x + e0 + g]);
      const int4 ax = __ldg(&P.aresd[gd.x + e0 + g]);
      uncut_block_row<DIM, NPE>(P, ax, ad.y & 255, P.D[ad.w], my, my + NPE * D2);
      z = (unsigned)ad.z;
    }
    reinterpret_cast<unsigned*>(my + NPE * D2 + DIM)[0] = z;
    __syncwarp(gmask);
    const int n_here = min(L, gd.y - e0);
    for (int s = g; s < nn; s += L) {
      double acc[D2];
#pragma unroll
      for (int i = 0; i < D2; ++i) acc[i] = slab[s * D2 + i];
      for (int j = 0; j < n_here; ++j) {
        const double* oj = scr + j * LD;
        const unsigned zj = reinterpret_cast<const unsigned*>(oj + NPE * D2 + DIM)[0];
#pragma unroll
        for (int b = 0; b < NPE; ++b)
          if (((zj >> (8 * b)) & 255u) == (unsigned)s)
#pragma unroll
            for (int i = 0; i < D2; ++i) acc[i] += oj[b * D2 + i];
      }
#pragma unroll
      for (int i = 0; i < D2; ++i) slab[s * D2 + i] = acc[i];
    }
    if (g == 0)
      for (int j = 0; j < n_here; ++j)
#pragma unroll
        for (int q = 0; q < DIM; ++q) rs[q] += scr[j * LD + NPE * D2 + q];
    __syncwarp(gmask);
  }
  const uint8_t* masks = P.dn_nbr_mask + gd.z;
  const int* pre = P.nbr_pre + gd.z;
  const int* rd = P.growd + (size_t)node * 3 * DIM;
#pragma unroll
  for (int q = 0; q < DIM; ++q) {
    const int gdof = __ldg(&rd[q]);
    const bool rf = gdof < P.n_free;
    if (P.flags & FLAG_JAC) {
      double* vF = P.val[rf ? 0 : 2] + __ldg(&rd[DIM + q]);
      double* vC = P.val[rf ? 1 : 3] + __ldg(&rd[2 * DIM + q]);
      for (int k = g; k < nn; k += L) {
        int pf = __ldg(&pre[k]);
        int pc = k * DIM - pf;
        const int mk = __ldg(&masks[k]);
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
          const double v = slab[(k * DIM + q) * DIM + d];
          if (mk & (1 << d)) vF[pf++] = v; else vC[pc++] = v;
        }
      }
    }
    if ((P.flags & FLAG_FUNC) && g == 0) {
      if (rf) P.Pf[gdof] = rs[q]; else P.Pp[gdof - P.n_free] = rs[q];
    }
  }
}

// Static residual of a general node for a group of L lanes (lane k of the group): the per-slot
// products of static_slot_product summed in slot order with shuffles, as static_resid_sum sums
// them, without the macroscale-strain response.  Every lane of the group gets the sum.
template <int DIM, int L>
__device__ __forceinline__ void static_resid_group(const DevProblem& P, int node, int nn, int k, unsigned gmask,
                                                   double* r) {
#pragma unroll
  for (int q = 0; q < DIM; ++q) r[q] = 0.0;
  const int s0 = __ldg(&P.stat_slot_off[node]);
  for (int k0 = 0; k0 < nn; k0 += L) {           // nn is uniform over the group
    double pk[DIM];
#pragma unroll
    for (int q = 0; q < DIM; ++q) pk[q] = 0.0;
    if (k0 + k < nn) static_slot_product<DIM>(P, s0, k0 + k, pk);
    const int n_here = min(L, nn - k0);
    for (int j = 0; j < n_here; ++j)
#pragma unroll
      for (int q = 0; q < DIM; ++q) r[q] += __shfl_sync(gmask, pk[q], j, L);
  }
}

// Residual-only rows of the general nodes, entry-parallel: L lanes per DOF node.  The node's
// static residual first (static blocks times displacements in slot order, then the macroscale-
// strain response), then lane k takes the node's entries k, k + L, ... and forms each entry's
// contribution (an uncut element's w B^T sigma; the cohesive traction at the node for a cut
// element the node is on a cohesive element of) -- the same operations general_rows performs --
// and the group adds the contributions in entry (adjacency) order with shuffles.  L divides 32.
template <int DIM, int L, int NPE = DIM + 1>
__global__ void __launch_bounds__(128) k_rows_general_resid(DevProblem P) {
  constexpr int NV = (DIM == 2) ? 3 : 6;
  constexpr int D2 = DIM * DIM;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int node = t / L, k = t % L;
  const bool valid = node < P.n_slow_dn;   // uniform over each group of L lanes
  const unsigned gmask = (L == 32) ? 0xffffffffu : (((1u << L) - 1u) << ((threadIdx.x & 31) / L * L));
  if (__all_sync(0xffffffffu, !valid)) return;
  int4 gd = make_int4(0, 0, 0, 0);
  if (valid) gd = __ldg(&P.gdesc[node]);
  double rs[DIM];
#pragma unroll
  for (int q = 0; q < DIM; ++q) rs[q] = 0.0;
  if (valid && node < P.n_stat) {                // uniform over the group
    static_resid_group<DIM, L>(P, node, gd.w, k, gmask, rs);
    if (P.subscale) {
      const double* Gs = P.stat_g + (size_t)node * DIM * NV;
#pragma unroll
      for (int q = 0; q < DIM; ++q)
#pragma unroll
        for (int v = 0; v < NV; ++v) rs[q] += __ldg(&Gs[q * NV + v]) * P.eps_macro[v];
    }
  }
  for (int e0 = 0; e0 < gd.y; e0 += L) {          // gd.y is uniform over the group
    const int ei = e0 + k;
    double re[DIM];
#pragma unroll
    for (int q = 0; q < DIM; ++q) re[q] = 0.0;
    if (ei < gd.y) {
      const int4 ad = __ldg(&P.adesc[gd.x + ei]);
      const int4 ax = __ldg(&P.aresd[gd.x + ei]);
      const int la = ad.y & 255, mn = ad.y >> 8;
      if (mn == 0) {
        double blk[NPE * D2];   // unused: the stiffness products are left to the compiler to drop
        uncut_block_row<DIM, NPE>(P, ax, la, P.D[ad.w], blk, re);
      } else if (ax.z >= 0) {
        coh_traction<DIM>(P, ax.z, re);
      }
    }
    // the node's sum in entry order
    const int n_here = min(L, gd.y - e0);
    for (int j = 0; j < n_here; ++j)
#pragma unroll
      for (int q = 0; q < DIM; ++q) rs[q] += __shfl_sync(gmask, re[q], j, L);
  }
  if (!valid || k >= DIM || !(P.flags & FLAG_FUNC)) return;
  double mine = rs[0];
#pragma unroll
  for (int q = 1; q < DIM; ++q) if (k == q) mine = rs[q];
  const int gdof = __ldg(&P.growd[(size_t)node * 3 * DIM + k]);
  if (gdof < P.n_free) P.Pf[gdof] = mine; else P.Pp[gdof - P.n_free] = mine;
}

// Set-up: the static part of the general rows (one thread per node of the image): each cut
// entry's volumetric block row (K_vol, from k_cut_volumetric) added into the node's neighbour
// slots and its macroscale-strain response into the node's sum, in entry order; in tri3 / tet4
// meshes the uncut elements' block rows and responses follow (every bulk law is linear elastic,
// so they do not depend on the state either), while quad4 meshes stop at the first uncut entry
// (the entries are cut-first).  stat and stat_g start at zero.
template <int DIM>
__global__ void __launch_bounds__(128) k_general_static(DevProblem P, double* stat, double* stat_g) {
  constexpr int NV = (DIM == 2) ? 3 : 6;
  constexpr int D2 = DIM * DIM;
  const int node = blockIdx.x * blockDim.x + threadIdx.x;
  if (node >= P.n_stat) return;
  const int4 gd = __ldg(&P.gdesc[node]);
  double* S = stat + (size_t)__ldg(&P.stat_slot_off[node]) * D2;
  double* Gs = stat_g + (size_t)node * DIM * NV;
  bool bad = false;
  for (int e = 0; e < gd.y; ++e) {
    const int4 ad = __ldg(&P.adesc[gd.x + e]);
    const int4 ax = __ldg(&P.aresd[gd.x + e]);
    const int la = ad.y & 255, mn = ad.y >> 8;
    if (mn == 0) {
      // uncut simplex (tri3 / tet4 meshes: every general node's image holds its uncut elements
      // too): the block row la, w B_la^T D B_b for each element node b, and the macroscale
      // response w B_la^T D -- the products of simplex_block, once per mesh
      if (P.npe != DIM + 1) break;
      constexpr int NPE = DIM + 1;
      const int nd[4] = {ax.x, ax.y, ax.z, ax.w};
      double x[NPE][DIM], g[NPE][DIM], J;
      for (int n = 0; n < NPE; ++n) load_node<DIM>(P.X, nd[n], x[n]);
      simplex_geom<DIM, double>(x, g, &J);
      const double wgt = J * ((DIM == 2) ? tri4_wsum() : tet5_wsum());
      const double* D = P.Dd + ad.w * 36;
      for (int q = 0; q < DIM; ++q) {
        double part[NV];
        bt_d_row<DIM, double>(D, g[la], q, part);
        for (int b = 0; b < NPE; ++b) {
          double* o = S + (size_t)((ad.z >> (8 * b)) & 255) * D2;
          for (int q2 = 0; q2 < DIM; ++q2) o[q * DIM + q2] += wgt * part_b<DIM, double>(part, g[b], q2);
        }
        for (int v = 0; v < NV; ++v) Gs[q * NV + v] += wgt * part[v];
      }
      continue;
    }
    const int cc = ax.x;
    const double* kr = P.ke + __ldg(&P.ke_off[cc]) + (size_t)la * mn * D2;   // block row la of K_vol
    for (int b = 0; b < mn; ++b) {
      double* o = S + (size_t)__ldg(&P.adj_slots[ad.z + b]) * D2;
#pragma unroll
      for (int i = 0; i < D2; ++i) o[i] += kr[b * D2 + i];
    }
    const double* gm = P.gmac + (size_t)__ldg(&P.re_off[cc]) / DIM * DIM * NV + (size_t)la * DIM * NV;
#pragma unroll
    for (int i = 0; i < DIM * NV; ++i) Gs[i] += gm[i];
  }
  for (int i = 0; i < gd.w * D2; ++i) bad |= !isfinite(S[i]);
  if (bad) atomicOr(P.err, ERR_NONFINITE);
}

// General rows of the nodes [node0, node1) of the general list.
template <int DIM, int L, int NPE = DIM + 1>
__global__ void __launch_bounds__(128) k_rows_general(DevProblem P, int slab_slots, int node0, int node1) {
  constexpr int NB = 128 / L;
  extern __shared__ double smem[];
  const int grp = threadIdx.x / L;
  const int node = node0 + blockIdx.x * NB + grp;
  general_rows<DIM, L, NPE>(P, node, node < node1,
                            smem + (size_t)grp * general_slab_doubles(slab_slots, DIM, L, NPE), slab_slots);
}

// Cohesive elements, one lane per quadrature point (CQ lanes per element: 2 in 2D for CohEdge2, 4
// in 3D for CohTri3 / CohQuad4).  Lane qi forms the opening delta = R sum_n N_n (U+ - U-) of its
// point, runs the traction-separation law with its internal-variable update and damage zone
// (src/Utilities.cpp:528-594, the Material_*Cohesive* files) and forms w R^T D R and w R^T T; the
// lanes then exchange these by shuffles and each writes some of the element's blocks
// B_ab = sum_qp N_a N_b w R^T D R (a, b < nh) and tractions t_a = sum_qp N_a w R^T T (sums in point
// order) to the scratch at kc_off[ce].  The element's stiffness block (n1, n2) is
// sgn * B_{n1 % nh, n2 % nh} and its internal force at n1 is sgn * t_{n1 % nh}, the signs following
// cohesiveKFast / cohesiveInternalForceFast.  Every lane of the warp must call it (valid = false
// for lanes past the last element).
template <int DIM>
struct CohLanes { static constexpr int CQ = (DIM == 2) ? 2 : 4; };

template <int DIM>
__device__ __forceinline__ void coh_element(const DevProblem& P, int ce, int qi, bool valid) {
  constexpr int D2 = DIM * DIM;
  constexpr int CQ = CohLanes<DIM>::CQ;
  const int lane = threadIdx.x & 31, base_lane = lane & ~(CQ - 1);
  int nh = 0, q0 = 0, nq = 0;
  if (valid) {
    nh = __ldg(&P.coh_nh[ce]);
    q0 = __ldg(&P.coh_qp_off[ce]);
    nq = min(CQ, __ldg(&P.coh_qp_off[ce + 1]) - q0);
  }
  double W[D2], Tr[DIM];
#pragma unroll
  for (int i = 0; i < D2; ++i) W[i] = 0.0;
#pragma unroll
  for (int i = 0; i < DIM; ++i) Tr[i] = 0.0;
  bool bad = false;
  if (valid && qi < nq) {
    const int* gn = P.coh_gnode + __ldg(&P.coh_local_off[ce]);   // the element's node ids
    const int cq = q0 + qi;
    const double* N = P.cqp_N + __ldg(&P.cqp_noff[cq]);
    const double* R = P.cqp_R + (size_t)cq * D2;
    double d0[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      double s = 0.0;
      for (int n = 0; n < nh; ++n) {
        const int np = __ldg(&gn[n + nh]), nm = __ldg(&gn[n]);
        s += N[n] * (P.U[(size_t)np * DIM + d] - P.U[(size_t)nm * DIM + d]);
      }
      d0[d] = s;
    }
    double dl[DIM], T[DIM], Dc[D2];
#pragma unroll
    for (int i = 0; i < DIM; ++i) {
      double s = 0.0;
#pragma unroll
      for (int j = 0; j < DIM; ++j) s += R[i * DIM + j] * d0[j];
      dl[i] = s;
    }
    const int iv = __ldg(&P.cqp_isv[cq]);
    double isv[2] = {0.0, 0.0};
    for (int v = 0; v < P.coh.nvar; ++v) isv[v] = P.isv_committed[iv + v];
    uint8_t z;
    coh_law(P.coh, DIM, dl, T, Dc, isv, &z);
    for (int v = 0; v < P.coh.nvar; ++v) P.isv_trial[iv + v] = isv[v];
    P.zone[cq] = z;
    double RtD[D2];
#pragma unroll
    for (int i = 0; i < DIM; ++i)
#pragma unroll
      for (int k = 0; k < DIM; ++k) {
        double s = 0.0;
#pragma unroll
        for (int j = 0; j < DIM; ++j) s += R[j * DIM + i] * Dc[j * DIM + k];
        RtD[i * DIM + k] = s;
      }
    const double w = P.cqp_wgt[cq];
#pragma unroll
    for (int i = 0; i < DIM; ++i)
#pragma unroll
      for (int l = 0; l < DIM; ++l) {
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < DIM; ++k) s += RtD[i * DIM + k] * R[k * DIM + l];
        W[i * DIM + l] = w * s;
        bad |= !isfinite(s);
      }
#pragma unroll
    for (int i = 0; i < DIM; ++i) {
      double s = 0.0;
#pragma unroll
      for (int j = 0; j < DIM; ++j) s += R[j * DIM + i] * T[j];
      Tr[i] = w * s;
      bad |= !isfinite(s);
    }
  }
  // every point's w R^T D R and w R^T T to every lane of the element
  double Wa[CQ][D2], Ta[CQ][DIM];
#pragma unroll
  for (int j = 0; j < CQ; ++j) {
#pragma unroll
    for (int i = 0; i < D2; ++i) Wa[j][i] = __shfl_sync(0xffffffffu, W[i], base_lane + j);
#pragma unroll
    for (int i = 0; i < DIM; ++i) Ta[j][i] = __shfl_sync(0xffffffffu, Tr[i], base_lane + j);
  }
  if (bad) atomicOr(P.err, ERR_NONFINITE);
  if (!valid) return;
  double* out = P.kcoh + __ldg(&P.kc_off[ce]);
  for (int p = qi; p < nh * nh; p += CQ) {
    const int a = p / nh, b = p - a * nh;
    double blk[D2];
#pragma unroll
    for (int i = 0; i < D2; ++i) blk[i] = 0.0;
#pragma unroll
    for (int j = 0; j < CQ; ++j) {
      if (j >= nq) break;
      const double* N = P.cqp_N + __ldg(&P.cqp_noff[q0 + j]);
      const double nn = N[a] * N[b];
#pragma unroll
      for (int i = 0; i < D2; ++i) blk[i] += nn * Wa[j][i];
    }
#pragma unroll
    for (int i = 0; i < D2; ++i) out[p * D2 + i] = blk[i];
  }
  for (int a = qi; a < nh; a += CQ) {
    double t[DIM];
#pragma unroll
    for (int i = 0; i < DIM; ++i) t[i] = 0.0;
#pragma unroll
    for (int j = 0; j < CQ; ++j) {
      if (j >= nq) break;
      const double na = P.cqp_N[__ldg(&P.cqp_noff[q0 + j]) + a];
#pragma unroll
      for (int i = 0; i < DIM; ++i) t[i] += na * Ta[j][i];
    }
#pragma unroll
    for (int i = 0; i < DIM; ++i) out[nh * nh * D2 + a * DIM + i] = t[i];
  }
}

template <int DIM>
__global__ void __launch_bounds__(128) k_coh_elements(DevProblem P) {
  constexpr int CQ = CohLanes<DIM>::CQ;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int ce = t / CQ;
  coh_element<DIM>(P, ce, t % CQ, ce < P.n_coh_el);
}

// State-independent part of the cut elements, computed once at set-up: the volumetric element
// matrix K_vol = sum over sub-element points of w B_i^T D B_j with the enriched gradients
// (src/Assembler.cpp:223-274; the bulk law is linear, so this block does not change between
// assemblies) and the macroscale-strain response G_i = sum w B_i^T D (R_i = K_vol,i U +
// G_i eps_macro).  One block per cut element, one thread per node pair; the element's gradients,
// weights and materials are staged in shared memory.  Blocks go to the cache in (i, j) block
// order so a block row is contiguous.  FP64.
__host__ __device__ inline int cut_smem_doubles(int nq, int mn, int dim) { return nq * mn * dim + 2 * nq + 3 * 36 + 8; }
template <int DIM>
__global__ void __launch_bounds__(64) k_cut_volumetric(DevProblem P, const int* __restrict__ list, int n_list, double* gmac) {
  constexpr int NV = (DIM == 2) ? 3 : 6;
  extern __shared__ double sm[];
  if ((int)blockIdx.x >= n_list) return;
  const int c = __ldg(&list[blockIdx.x]);
  const int mn = __ldg(&P.cut_node_off[c + 1]) - __ldg(&P.cut_node_off[c]);
  const int q0 = __ldg(&P.cut_qp_off[c]), q1 = __ldg(&P.cut_qp_off[c + 1]);
  const int nq = q1 - q0;
  double* sg = sm;
  double* sw = sg + (size_t)nq * mn * DIM;
  double* smat = sw + nq;
  double* sD = smat + nq;
  const int gbase = __ldg(&P.qp_grad_off[q0]);
  for (int i = threadIdx.x; i < nq * mn * DIM; i += blockDim.x) sg[i] = __ldg(&P.qp_grad[gbase + i]);
  for (int i = threadIdx.x; i < nq; i += blockDim.x) { sw[i] = __ldg(&P.qp_wgt[q0 + i]); smat[i] = (double)__ldg(&P.qp_mat[q0 + i]); }
  for (int i = threadIdx.x; i < 108; i += blockDim.x) sD[i] = __ldg(&P.Dd[i]);
  __syncthreads();
  double* kout = P.ke + __ldg(&P.ke_off[c]);
  bool bad = false;
  for (int p = threadIdx.x; p < mn * mn; p += blockDim.x) {
    const int i = p / mn, j = p - i * mn;
    double kb[DIM][DIM];
#pragma unroll
    for (int x = 0; x < DIM; ++x)
#pragma unroll
      for (int y = 0; y < DIM; ++y) kb[x][y] = 0.0;
    for (int qq = 0; qq < nq; ++qq) {
      const double w = sw[qq];
      const double* D = sD + 36 * (int)smat[qq];
      const double* gi = sg + ((size_t)qq * mn + i) * DIM;
      const double* gj = sg + ((size_t)qq * mn + j) * DIM;
#pragma unroll
      for (int q = 0; q < DIM; ++q) {
        double part[NV];
        bt_d_row<DIM, double>(D, gi, q, part);
#pragma unroll
        for (int q2 = 0; q2 < DIM; ++q2) kb[q][q2] += w * part_b<DIM, double>(part, gj, q2);
      }
    }
    double* o = kout + (size_t)p * DIM * DIM;
#pragma unroll
    for (int x = 0; x < DIM; ++x)
#pragma unroll
      for (int y = 0; y < DIM; ++y) { o[x * DIM + y] = kb[x][y]; bad |= !isfinite(kb[x][y]); }
  }
  double* gout = gmac + (size_t)__ldg(&P.re_off[c]) / DIM * DIM * NV;
  for (int i = threadIdx.x; i < mn; i += blockDim.x) {
    double gacc[DIM][NV];
#pragma unroll
    for (int q = 0; q < DIM; ++q)
#pragma unroll
      for (int v = 0; v < NV; ++v) gacc[q][v] = 0.0;
    for (int qq = 0; qq < nq; ++qq) {
      const double* gi = sg + ((size_t)qq * mn + i) * DIM;
      const double* D = sD + 36 * (int)smat[qq];
#pragma unroll
      for (int q = 0; q < DIM; ++q) {
        double part[NV];
        bt_d_row<DIM, double>(D, gi, q, part);
#pragma unroll
        for (int v = 0; v < NV; ++v) gacc[q][v] += sw[qq] * part[v];
      }
    }
#pragma unroll
    for (int q = 0; q < DIM; ++q)
#pragma unroll
      for (int v = 0; v < NV; ++v) gout[((size_t)i * DIM + q) * NV + v] = gacc[q][v];
  }
  if (bad) atomicOr(P.err, ERR_NONFINITE);
}

}  // namespace pgd
