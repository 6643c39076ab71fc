// pg_kernels.cuh -- the assembly kernels.
//
//   k_coh_points     one thread per cohesive quadrature point: opening delta = R sum_n N_n (U+ - U-),
//                    the traction-separation law with its internal-variable update and damage
//                    zone, and the weighted R^T D R / R^T T (src/Utilities.cpp:528-594).  FP64.
//   k_cut_volumetric run once at set-up: the cut elements' volumetric (linear, state-independent)
//                    element matrices from sub-element quadrature with enriched B-matrices
//                    (src/Assembler.cpp:223-274), cached for every later assembly.  FP64.
//   k_rows_general   one lane group per DOF node (row owner) for every node the structured stencil
//                    path (pg_stencil.cuh) does not take: boundary rows, nodes of cut elements and
//                    enrichment nodes; uncut elements are recomputed from node coordinates; for cut
//                    elements the cached volumetric block row is combined with the nodal
//                    displacements and the cohesive points' blocks (src/Assembler.cpp:278-365).
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

// Block row of an uncut simplex for local node la: kv[lb][q][q2] = w (B_la^T D B_lb)[q][q2],
// rv[q] = w (B_la^T sigma)[q].
template <int DIM, typename T>
__device__ __forceinline__ void simplex_block_row(const DevProblem& P, int e, int la, const T* D, T (*kv)[DIM][DIM], T* rv) {
  constexpr int NPE = DIM + 1;
  constexpr int NV = (DIM == 2) ? 3 : 6;
  int nd[NPE];
#pragma unroll
  for (int n = 0; n < NPE; ++n) nd[n] = __ldg(&P.conn[(size_t)e * NPE + n]);
  T x[NPE][DIM], u[NPE][DIM], g[NPE][DIM], J;
#pragma unroll
  for (int n = 0; n < NPE; ++n)
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      if (sizeof(T) == 4) x[n][d] = (T)__ldg(&P.Xf[(size_t)nd[n] * DIM + d]);
      else x[n][d] = (T)__ldg(&P.X[(size_t)nd[n] * DIM + d]);
      u[n][d] = (T)__ldg(&P.U[(size_t)nd[n] * DIM + d]);
    }
  simplex_geom<DIM, T>(x, g, &J);
  const T wgt = J * (T)((DIM == 2) ? tri4_wsum() : tet5_wsum());
  T eps[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) eps[v] = 0;
#pragma unroll
  for (int n = 0; n < NPE; ++n) add_strain<DIM, T>(g[n], u[n], eps);
  if (P.subscale) {
#pragma unroll
    for (int v = 0; v < NV; ++v) eps[v] += (T)P.eps_macro[v];
  }
  T sig[NV];
  lei_stress<DIM, T>(D, eps, sig);
  // la is a runtime index: copy its gradient once
  T ga[DIM];
#pragma unroll
  for (int d = 0; d < DIM; ++d) ga[d] = g[0][d];
#pragma unroll
  for (int n = 1; n < NPE; ++n)
    if (la == n)
#pragma unroll
      for (int d = 0; d < DIM; ++d) ga[d] = g[n][d];
#pragma unroll
  for (int q = 0; q < DIM; ++q) {
    T part[NV];
    bt_d_row<DIM, T>(D, ga, q, part);
    rv[q] = wgt * bt_sig<DIM, T>(ga, sig, q);
#pragma unroll
    for (int lb = 0; lb < NPE; ++lb)
#pragma unroll
      for (int q2 = 0; q2 < DIM; ++q2) kv[lb][q][q2] = wgt * part_b<DIM, T>(part, g[lb], q2);
  }
}

// Row assembly for the DOF nodes the stencil path does not take (boundary rows, nodes of cut
// elements, enrichment nodes): one lane group of G threads per DOF node.  Each lane takes one
// adjacent element (uncut: geometry recomputed from the node coordinates; cut: its block row from
// the scratch), the lanes add their block rows into the node's shared-memory slab one after
// another in adjacency order (deterministic, no atomics), the residual is reduced with a fixed
// shuffle tree, and the group writes every CSR value of the node's rows exactly once.
// Everything a node or an adjacency entry needs is packed into descriptors so the dependent
// loads are: node descriptor -> adjacency descriptors -> element data.
//   gdesc[node]      int4 {adjacency begin, adjacency count, neighbour begin, neighbour count}
//   growd[node]      3*DIM ints: global DOF of each row, first slot in the row's F block, in its C block
//   adesc[entry]     int4 {element, local node | nodes of a cut element << 8, slots (uncut: 8 bits per
//                    node; cut: offset into adj_slots), material (uncut) / block-row offset (cut)}
//   aresd[entry]     element-vector offset of the cut element's row (cut entries)
// Shared-memory doubles of one lane group's slab: slab_slots blocks of DIM x DIM plus the node's
// residual (4 doubles reserved).
__host__ __device__ inline int general_slab_doubles(int slab_slots, int dim) { return slab_slots * dim * dim + 4; }

// Rows of general node `node` (an index into the general-node descriptors) for the lane group of
// the calling thread (G lanes, 128 / G groups per 128-thread block).  Every lane of the warp must
// call it (valid = false for lanes without a node) because of the warp-wide shuffles.  slab: this
// group's shared-memory slab of general_slab_doubles(slab_slots, DIM) doubles.  The K blocks and
// the residual are both summed over the adjacent elements in adjacency order, one lane after
// another, so the result does not depend on G.
template <int DIM, int G>
__device__ __forceinline__ void general_rows(const DevProblem& P, int node, bool valid, double* slab) {
  constexpr int NPE = DIM + 1;
  constexpr int NV = (DIM == 2) ? 3 : 6;
  const int g = threadIdx.x % G;
  int4 gd = make_int4(0, 0, 0, 0);
  double* rs = nullptr;   // the node's residual, after the slab blocks
  if (valid) {
    gd = __ldg(&P.gdesc[node]);
    rs = slab + gd.w * DIM * DIM;
    for (int i = g; i < gd.w * DIM * DIM + DIM; i += G) slab[i] = 0.0;
  }
  int passes = (gd.y + G - 1) / G;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) passes = max(passes, __shfl_xor_sync(0xffffffffu, passes, o));
  __syncwarp();
  for (int pass = 0; pass < passes; ++pass) {
    const int idx = pass * G + g;
    const bool have = valid && idx < gd.y;
    int4 ad = make_int4(0, 0, 0, 0);
    double kv[NPE][DIM][DIM];
    double r[DIM];   // this entry's residual contribution
#pragma unroll
    for (int q = 0; q < DIM; ++q) r[q] = 0.0;
    if (have) {
      ad = __ldg(&P.adesc[gd.x + idx]);
      const int la = ad.y & 255, mn = ad.y >> 8;
      if (mn == 0) {
        double D[NV * NV];
#pragma unroll
        for (int i = 0; i < NV * NV; ++i) D[i] = __ldg(&P.Dd[ad.w * 36 + i]);
        double rv[DIM];
        simplex_block_row<DIM, double>(P, ad.x, la, D, kv, rv);
#pragma unroll
        for (int q = 0; q < DIM; ++q) r[q] += rv[q];
      } else {
        // cut element: K_vol (state independent, cached at set-up) times the element's nodal
        // displacements, the macroscale-strain response, and the cohesive internal forces
        const int cc = __ldg(&P.aresd[gd.x + idx]);
        const double* kb = P.ke + ad.w;
        const int* cn = P.cut_nodes + __ldg(&P.cut_node_off[cc]);
        for (int lb = 0; lb < mn; ++lb) {
          const int nd = __ldg(&cn[lb]);
          double u[DIM];
#pragma unroll
          for (int d = 0; d < DIM; ++d) u[d] = P.U[(size_t)nd * DIM + d];
#pragma unroll
          for (int q = 0; q < DIM; ++q)
#pragma unroll
            for (int d = 0; d < DIM; ++d) r[q] += kb[lb * DIM * DIM + q * DIM + d] * u[d];
        }
        if (P.subscale) {
          const double* gm = P.gmac + __ldg(&P.re_off[cc]) / DIM * DIM * NV + (size_t)la * DIM * NV;
#pragma unroll
          for (int q = 0; q < DIM; ++q)
#pragma unroll
            for (int v = 0; v < NV; ++v) r[q] += gm[q * NV + v] * P.eps_macro[v];
        }
        const int ce0 = __ldg(&P.cut_coh_off[cc]), ce1 = __ldg(&P.cut_coh_off[cc + 1]);
        for (int ce = ce0; ce < ce1; ++ce) {
          const int nh = __ldg(&P.coh_nh[ce]);
          const int* cl = P.coh_local + __ldg(&P.coh_local_off[ce]);
          int n1 = -1;
          for (int k = 0; k < 2 * nh; ++k) if (__ldg(&cl[k]) == la) n1 = k;
          if (n1 < 0) continue;
          const double sgn = (n1 >= nh) ? 1.0 : -1.0;
          double pc[DIM];
#pragma unroll
          for (int d = 0; d < DIM; ++d) pc[d] = 0.0;
          for (int cq = __ldg(&P.coh_qp_off[ce]); cq < __ldg(&P.coh_qp_off[ce + 1]); ++cq) {
            const double nv = __ldg(&P.cqp_N[__ldg(&P.cqp_noff[cq]) + n1 % nh]);
            const double* wt = P.cpt + (size_t)cq * (DIM * DIM + DIM) + DIM * DIM;
#pragma unroll
            for (int d = 0; d < DIM; ++d) pc[d] += sgn * (nv * wt[d]);
          }
#pragma unroll
          for (int d = 0; d < DIM; ++d) r[d] += pc[d];
        }
      }
    }
    for (int t = 0; t < G; ++t) {
      if (have && g == t) {
#pragma unroll
        for (int q = 0; q < DIM; ++q) rs[q] += r[q];
        const int mn = ad.y >> 8;
        if (mn == 0) {
          const unsigned slots = (unsigned)ad.z;
#pragma unroll
          for (int lb = 0; lb < NPE; ++lb) {
            double* ak = slab + ((slots >> (8 * lb)) & 255) * DIM * DIM;
#pragma unroll
            for (int i = 0; i < DIM * DIM; ++i) ak[i] += kv[lb][i / DIM][i % DIM];
          }
        } else {
          const double* kb = P.ke + ad.w;
          for (int lb = 0; lb < mn; ++lb) {
            double* ak = slab + __ldg(&P.adj_slots[ad.z + lb]) * DIM * DIM;
#pragma unroll
            for (int i = 0; i < DIM * DIM; ++i) ak[i] += kb[lb * DIM * DIM + i];
          }
          // cohesive blocks: sgn N_a1 N_a2 (w R^T D R) summed over the cohesive element's points
          const int la = ad.y & 255;
          const int cc = __ldg(&P.aresd[gd.x + idx]);
          const int ce0 = __ldg(&P.cut_coh_off[cc]), ce1 = __ldg(&P.cut_coh_off[cc + 1]);
          for (int ce = ce0; ce < ce1; ++ce) {
            const int nh = __ldg(&P.coh_nh[ce]);
            const int* cl = P.coh_local + __ldg(&P.coh_local_off[ce]);
            int n1 = -1;
            for (int k = 0; k < 2 * nh; ++k) if (__ldg(&cl[k]) == la) n1 = k;
            if (n1 < 0) continue;
            const int cqa = __ldg(&P.coh_qp_off[ce]), cqb = __ldg(&P.coh_qp_off[ce + 1]);
            for (int n2 = 0; n2 < 2 * nh; ++n2) {
              const double sgn = ((n1 >= nh) == (n2 >= nh)) ? 1.0 : -1.0;
              double kc[DIM * DIM];
#pragma unroll
              for (int i = 0; i < DIM * DIM; ++i) kc[i] = 0.0;
              for (int cq = cqa; cq < cqb; ++cq) {
                const int no = __ldg(&P.cqp_noff[cq]);
                const double nn = __ldg(&P.cqp_N[no + n1 % nh]) * __ldg(&P.cqp_N[no + n2 % nh]);
                const double* wr = P.cpt + (size_t)cq * (DIM * DIM + DIM);
#pragma unroll
                for (int i = 0; i < DIM * DIM; ++i) kc[i] += sgn * (nn * wr[i]);
              }
              double* ak = slab + __ldg(&P.adj_slots[ad.z + __ldg(&cl[n2])]) * DIM * DIM;
#pragma unroll
              for (int i = 0; i < DIM * DIM; ++i) ak[i] += kc[i];
            }
          }
        }
      }
      __syncwarp();
    }
  }
  if (!valid) return;
  const int nn = gd.w;
  const uint8_t* masks = P.dn_nbr_mask + gd.z;
  const int* rd = P.growd + (size_t)node * 3 * DIM;
#pragma unroll
  for (int q = 0; q < DIM; ++q) {
    const int gdof = __ldg(&rd[q]);
    const bool rf = gdof < P.n_free;
    if (P.flags & FLAG_JAC) {
      double* vF = P.val[rf ? 0 : 2] + __ldg(&rd[DIM + q]);
      double* vC = P.val[rf ? 1 : 3] + __ldg(&rd[2 * DIM + q]);
      for (int k = g; k < nn; k += G) {
        int pf = 0;
        for (int k2 = 0; k2 < k; ++k2) pf += __popc(__ldg(&masks[k2]));
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

template <int DIM, int G>
__global__ void __launch_bounds__(128) k_rows_general(DevProblem P, int slab_slots) {
  constexpr int NB = 128 / G;
  extern __shared__ double smem[];
  const int grp = threadIdx.x / G;
  const int node = blockIdx.x * NB + grp;
  general_rows<DIM, G>(P, node, node < P.n_slow_dn, smem + (size_t)grp * general_slab_doubles(slab_slots, DIM));
}

// Cohesive law at every cohesive quadrature point.  Output per point: w R^T D R (dim x dim) then
// w R^T T (dim).
template <int DIM>
__device__ __forceinline__ void coh_point(const DevProblem& P, int cq) {
  const int c = __ldg(&P.cqp_cut[cq]), ce = __ldg(&P.cqp_ce[cq]);
  const int nh = __ldg(&P.coh_nh[ce]);
  const int* cl = P.coh_local + __ldg(&P.coh_local_off[ce]);
  const int* nodes = P.cut_nodes + __ldg(&P.cut_node_off[c]);
  const double* N = P.cqp_N + __ldg(&P.cqp_noff[cq]);
  const double* R = P.cqp_R + (size_t)cq * DIM * DIM;
  double d0[DIM];
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    double s = 0.0;
    for (int n = 0; n < nh; ++n) {
      const int np = __ldg(&nodes[__ldg(&cl[n + nh])]), nm = __ldg(&nodes[__ldg(&cl[n])]);
      s += N[n] * (P.U[(size_t)np * DIM + d] - P.U[(size_t)nm * DIM + d]);
    }
    d0[d] = s;
  }
  double dl[DIM], T[DIM], Dc[DIM * DIM];
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
  double RtD[DIM * DIM];
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
  double* out = P.cpt + (size_t)cq * (DIM * DIM + DIM);
  bool bad = false;
#pragma unroll
  for (int i = 0; i < DIM; ++i)
#pragma unroll
    for (int l = 0; l < DIM; ++l) {
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < DIM; ++k) s += RtD[i * DIM + k] * R[k * DIM + l];
      out[i * DIM + l] = w * s;
      bad |= !isfinite(s);
    }
#pragma unroll
  for (int i = 0; i < DIM; ++i) {
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < DIM; ++j) s += R[j * DIM + i] * T[j];
    out[DIM * DIM + i] = w * s;
    bad |= !isfinite(s);
  }
  if (bad) atomicOr(P.err, ERR_NONFINITE);
}

template <int DIM>
__global__ void __launch_bounds__(128) k_coh_points(DevProblem P) {
  const int cq = blockIdx.x * blockDim.x + threadIdx.x;
  if (cq < P.n_coh_qp) coh_point<DIM>(P, cq);
}

// State-independent part of the cut elements, computed once at set-up: the volumetric element
// matrix K_vol = sum over sub-element points of w B_i^T D B_j with the enriched gradients
// (src/Assembler.cpp:223-274; the bulk law is linear, so this block does not change between
// assemblies) and the macroscale-strain response G_i = sum w B_i^T D (R_i = K_vol,i U +
// G_i eps_macro).  One block per cut element, one thread per node pair; the element's gradients,
// weights and materials are staged in shared memory.  Blocks go to the cache in (i, j) block
// order so a block row is contiguous.  FP64.
__host__ __device__ inline int cut_smem_doubles(int nq, int mn, int dim) { return nq * mn * dim + 2 * nq + 2 * 36 + 8; }
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
  for (int i = threadIdx.x; i < 72; i += blockDim.x) sD[i] = __ldg(&P.Dd[i]);
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
