// pg_kernels.cuh -- the assembly kernels.
//
//   k_coh_points     one thread per cohesive quadrature point: opening delta = R sum_n N_n (U+ - U-)
//                    (src/Utilities.cpp:528-540), the traction-separation law with its internal-
//                    variable update and damage zone, and the weighted R^T D R / R^T T the element
//                    blocks need (src/Utilities.cpp:543-594).  FP64.
//   k_cut_blocks     one block per cut element, one thread per node pair (i, j): the dim x dim
//                    block of the element matrix, sum over sub-element quadrature points of
//                    w B_i^T D B_j with enriched gradients (src/Assembler.cpp:223-274) plus the
//                    cohesive blocks (src/Assembler.cpp:278-365); one thread per node for the
//                    element vector.  Blocks go to a scratch area in (i, j) block order so a block
//                    row is contiguous.  FP64.
//   k_rows_fast      one thread per DOF node whose elements are all uncut simplices: recomputes the
//                    geometry of each adjacent element from node coordinates, accumulates its block
//                    row in a per-thread shared-memory slab (one dim x dim block per neighbour node,
//                    slots precomputed), then writes every CSR value of its dim rows exactly once,
//                    plus the residual entries.  Runs concurrently with the cut-element kernels.
//   k_rows_general   the same ownership for the remaining DOF nodes (nodes of cut elements,
//                    enrichment nodes), taking cut-element block rows from the scratch.
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

// Writes the dim rows of DOF node a from the slab acc (slot-major, dim x dim per slot).
template <int DIM>
__device__ __forceinline__ void write_rows(const DevProblem& P, int a, int nn, const double* acc, int stride, const double* r) {
  const int na = __ldg(&P.dn_node[a]);
  const int nb0 = __ldg(&P.dn_nbr_off[a]);
#pragma unroll
  for (int q = 0; q < DIM; ++q) {
    const int gdof = __ldg(&P.node_dof[(size_t)na * DIM + q]);
    const bool rf = gdof < P.n_free;
    const int rr = rf ? gdof : gdof - P.n_free;
    if (P.flags & FLAG_JAC) {
      const int bF = rf ? 0 : 2, bC = rf ? 1 : 3;
      double* vF = P.val[bF] + __ldg(&P.rp[bF][rr]);
      double* vC = P.val[bC] + __ldg(&P.rp[bC][rr]);
      for (int k = 0; k < nn; ++k) {
        const int mask = __ldg(&P.dn_nbr_mask[nb0 + k]);
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
          const double v = acc[((k * DIM + q) * DIM + d) * stride];
          if (mask & (1 << d)) *vF++ = v; else *vC++ = v;
        }
      }
    }
    if (P.flags & FLAG_FUNC) {
      if (rf) P.Pf[rr] = r[q]; else P.Pp[rr] = r[q];
    }
  }
}

// DOF nodes whose adjacent elements are all uncut simplices.  acc: MAXNB x dim x dim doubles per
// thread in shared memory, thread-interleaved (stride = blockDim.x) so lanes hit distinct banks.
template <int DIM, int MAXNB, typename T>
__global__ void __launch_bounds__(128) k_rows_fast(DevProblem P) {
  constexpr int NPE = DIM + 1;
  constexpr int NV = (DIM == 2) ? 3 : 6;
  extern __shared__ double slab[];
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= P.n_fast_dn) return;
  const int stride = blockDim.x;
  double* acc = slab + threadIdx.x;
  const int a = __ldg(&P.fast_dn[t]);
  const int nn = __ldg(&P.dn_nbr_off[a + 1]) - __ldg(&P.dn_nbr_off[a]);
  for (int i = 0; i < nn * DIM * DIM; ++i) acc[i * stride] = 0.0;
  T D[2][NV * NV];
#pragma unroll
  for (int m = 0; m < 2; ++m)
#pragma unroll
    for (int i = 0; i < NV * NV; ++i) D[m][i] = (sizeof(T) == 4) ? (T)P.Df[m][i] : (T)P.D[m][i];
  double r[DIM];
#pragma unroll
  for (int q = 0; q < DIM; ++q) r[q] = 0.0;
  const int ad0 = __ldg(&P.dn_adj_off[a]), ad1 = __ldg(&P.dn_adj_off[a + 1]);
  for (int s = ad0; s < ad1; ++s) {
    const int ent = __ldg(&P.dn_adj[s]);
    const unsigned slots = (unsigned)__ldg(&P.adj_slot32[s]);
    const int e = ent >> 5, la = ent & 31;
    const int m = __ldg(&P.emat[e]);
    T kv[NPE][DIM][DIM], rv[DIM];
    simplex_block_row<DIM, T>(P, e, la, m ? D[1] : D[0], kv, rv);
#pragma unroll
    for (int q = 0; q < DIM; ++q) r[q] += (double)rv[q];
#pragma unroll
    for (int lb = 0; lb < NPE; ++lb) {
      const int k = (slots >> (8 * lb)) & 255;
      double* ak = acc + (size_t)k * DIM * DIM * stride;
#pragma unroll
      for (int q = 0; q < DIM; ++q)
#pragma unroll
        for (int d = 0; d < DIM; ++d) ak[(q * DIM + d) * stride] += (double)kv[lb][q][d];
    }
  }
  write_rows<DIM>(P, a, nn, acc, stride, r);
}

// Remaining DOF nodes; the slab holds P.maxnb_general slots per thread.
template <int DIM>
__global__ void __launch_bounds__(64) k_rows_general(DevProblem P) {
  constexpr int NPE = DIM + 1;
  extern __shared__ double slab[];
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= P.n_slow_dn) return;
  const int stride = blockDim.x;
  double* acc = slab + threadIdx.x;
  const int a = __ldg(&P.slow_dn[t]);
  const int nn = __ldg(&P.dn_nbr_off[a + 1]) - __ldg(&P.dn_nbr_off[a]);
  for (int i = 0; i < nn * DIM * DIM; ++i) acc[i * stride] = 0.0;
  double r[DIM];
#pragma unroll
  for (int q = 0; q < DIM; ++q) r[q] = 0.0;
  const int ad0 = __ldg(&P.dn_adj_off[a]), ad1 = __ldg(&P.dn_adj_off[a + 1]);
  for (int s = ad0; s < ad1; ++s) {
    const int ent = __ldg(&P.dn_adj[s]);
    const int e = ent >> 5, la = ent & 31;
    const int c = __ldg(&P.cut_of[e]);
    if (c < 0) {
      const unsigned slots = (unsigned)__ldg(&P.adj_slot32[s]);
      const int m = __ldg(&P.emat[e]);
      double kv[NPE][DIM][DIM], rv[DIM];
      simplex_block_row<DIM, double>(P, e, la, P.D[m], kv, rv);
#pragma unroll
      for (int q = 0; q < DIM; ++q) r[q] += rv[q];
#pragma unroll
      for (int lb = 0; lb < NPE; ++lb) {
        const int k = (slots >> (8 * lb)) & 255;
        double* ak = acc + (size_t)k * DIM * DIM * stride;
#pragma unroll
        for (int q = 0; q < DIM; ++q)
#pragma unroll
          for (int d = 0; d < DIM; ++d) ak[(q * DIM + d) * stride] += kv[lb][q][d];
      }
    } else {
      const int mn = __ldg(&P.cut_node_off[c + 1]) - __ldg(&P.cut_node_off[c]);
      const double* kb = P.ke + __ldg(&P.ke_off[c]) + (size_t)la * mn * DIM * DIM;
      const double* rb = P.re + __ldg(&P.re_off[c]) + la * DIM;
#pragma unroll
      for (int q = 0; q < DIM; ++q) r[q] += rb[q];
      const int so = __ldg(&P.adj_slot_off[s]);
      for (int lb = 0; lb < mn; ++lb) {
        const int k = __ldg(&P.adj_slots[so + lb]);
        double* ak = acc + (size_t)k * DIM * DIM * stride;
#pragma unroll
        for (int i = 0; i < DIM * DIM; ++i) ak[i * stride] += kb[lb * DIM * DIM + i];
      }
    }
  }
  write_rows<DIM>(P, a, nn, acc, stride, r);
}

// Cohesive law at every cohesive quadrature point.  Output per point: w R^T D R (dim x dim) then
// w R^T T (dim).
template <int DIM>
__global__ void __launch_bounds__(128) k_coh_points(DevProblem P) {
  const int cq = blockIdx.x * blockDim.x + threadIdx.x;
  if (cq >= P.n_coh_qp) return;
  const int c = __ldg(&P.cqp_cut[cq]), ce = __ldg(&P.cqp_ce[cq]);
  const int nh = __ldg(&P.coh_nh[ce]);
  const int* cl = P.coh_local + __ldg(&P.coh_local_off[ce]);
  const int* nodes = P.cut_nodes + __ldg(&P.cut_node_off[c]);
  const double* N = P.cqp_N + (size_t)cq * nh;
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

// Element blocks of the cut elements (see the file comment).
template <int DIM>
__global__ void __launch_bounds__(64) k_cut_blocks(DevProblem P) {
  constexpr int NV = (DIM == 2) ? 3 : 6;
  const int c = blockIdx.x;
  if (c >= P.ncut) return;
  const int o0 = __ldg(&P.cut_node_off[c]);
  const int mn = __ldg(&P.cut_node_off[c + 1]) - o0;
  const int q0 = __ldg(&P.cut_qp_off[c]), q1 = __ldg(&P.cut_qp_off[c + 1]);
  const int ce0 = __ldg(&P.cut_coh_off[c]), ce1 = __ldg(&P.cut_coh_off[c + 1]);
  double* kout = P.ke + __ldg(&P.ke_off[c]);
  bool bad = false;
  for (int p = threadIdx.x; p < mn * mn; p += blockDim.x) {
    const int i = p / mn, j = p - i * mn;
    double kb[DIM][DIM];
#pragma unroll
    for (int a = 0; a < DIM; ++a)
#pragma unroll
      for (int b = 0; b < DIM; ++b) kb[a][b] = 0.0;
    for (int qp = q0; qp < q1; ++qp) {
      const double w = __ldg(&P.qp_wgt[qp]);
      const double* D = P.D[__ldg(&P.qp_mat[qp])];
      const double* g = P.qp_grad + __ldg(&P.qp_grad_off[qp]);
      double gi[DIM], gj[DIM];
#pragma unroll
      for (int d = 0; d < DIM; ++d) { gi[d] = __ldg(&g[i * DIM + d]); gj[d] = __ldg(&g[j * DIM + d]); }
#pragma unroll
      for (int q = 0; q < DIM; ++q) {
        double part[NV];
        bt_d_row<DIM, double>(D, gi, q, part);
#pragma unroll
        for (int q2 = 0; q2 < DIM; ++q2) kb[q][q2] += w * part_b<DIM, double>(part, gj, q2);
      }
    }
    for (int ce = ce0; ce < ce1; ++ce) {
      const int nh = __ldg(&P.coh_nh[ce]);
      const int* cl = P.coh_local + __ldg(&P.coh_local_off[ce]);
      int n1 = -1, n2 = -1;
      for (int k = 0; k < 2 * nh; ++k) {
        const int v = __ldg(&cl[k]);
        if (v == i) n1 = k;
        if (v == j) n2 = k;
      }
      if (n1 < 0 || n2 < 0) continue;
      const int a1 = n1 % nh, a2 = n2 % nh;
      const double sgn = ((n1 >= nh) == (n2 >= nh)) ? 1.0 : -1.0;
      const int cq0 = __ldg(&P.coh_qp_off[ce]), cq1 = __ldg(&P.coh_qp_off[ce + 1]);
      for (int cq = cq0; cq < cq1; ++cq) {
        const double* N = P.cqp_N + (size_t)cq * nh;
        const double* wr = P.cpt + (size_t)cq * (DIM * DIM + DIM);
        const double nn = N[a1] * N[a2];
#pragma unroll
        for (int a = 0; a < DIM; ++a)
#pragma unroll
          for (int b = 0; b < DIM; ++b) kb[a][b] += sgn * (nn * wr[a * DIM + b]);
      }
    }
    double* o = kout + (size_t)p * DIM * DIM;
#pragma unroll
    for (int a = 0; a < DIM; ++a)
#pragma unroll
      for (int b = 0; b < DIM; ++b) { o[a * DIM + b] = kb[a][b]; bad |= !isfinite(kb[a][b]); }
  }
  // element vector: one thread per node
  const int* nodes = P.cut_nodes + o0;
  for (int i = threadIdx.x; i < mn; i += blockDim.x) {
    double r[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) r[d] = 0.0;
    for (int qp = q0; qp < q1; ++qp) {
      const double w = __ldg(&P.qp_wgt[qp]);
      const double* D = P.D[__ldg(&P.qp_mat[qp])];
      const double* g = P.qp_grad + __ldg(&P.qp_grad_off[qp]);
      double eps[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) eps[v] = 0.0;
      for (int n = 0; n < mn; ++n) {
        const int nd = __ldg(&nodes[n]);
        double gn[DIM], un[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) { gn[d] = __ldg(&g[n * DIM + d]); un[d] = P.U[(size_t)nd * DIM + d]; }
        add_strain<DIM, double>(gn, un, eps);
      }
      if (P.subscale) {
#pragma unroll
        for (int v = 0; v < NV; ++v) eps[v] += P.eps_macro[v];
      }
      double sig[NV];
      lei_stress<DIM, double>(D, eps, sig);
      double gi[DIM];
#pragma unroll
      for (int d = 0; d < DIM; ++d) gi[d] = __ldg(&g[i * DIM + d]);
#pragma unroll
      for (int q = 0; q < DIM; ++q) r[q] += w * bt_sig<DIM, double>(gi, sig, q);
    }
    for (int ce = ce0; ce < ce1; ++ce) {
      const int nh = __ldg(&P.coh_nh[ce]);
      const int* cl = P.coh_local + __ldg(&P.coh_local_off[ce]);
      int n1 = -1;
      for (int k = 0; k < 2 * nh; ++k) if (__ldg(&cl[k]) == i) n1 = k;
      if (n1 < 0) continue;
      const double sgn = (n1 >= nh) ? 1.0 : -1.0;
      const int cq0 = __ldg(&P.coh_qp_off[ce]), cq1 = __ldg(&P.coh_qp_off[ce + 1]);
      double pc[DIM];
#pragma unroll
      for (int d = 0; d < DIM; ++d) pc[d] = 0.0;
      for (int cq = cq0; cq < cq1; ++cq) {
        const double* N = P.cqp_N + (size_t)cq * nh;
        const double* wt = P.cpt + (size_t)cq * (DIM * DIM + DIM) + DIM * DIM;
#pragma unroll
        for (int d = 0; d < DIM; ++d) pc[d] += sgn * (N[n1 % nh] * wt[d]);
      }
#pragma unroll
      for (int d = 0; d < DIM; ++d) r[d] += pc[d];
    }
    double* ro = P.re + __ldg(&P.re_off[c]) + i * DIM;
#pragma unroll
    for (int d = 0; d < DIM; ++d) { ro[d] = r[d]; bad |= !isfinite(r[d]); }
  }
  if (bad) atomicOr(P.err, ERR_NONFINITE);
}

}  // namespace pgd
