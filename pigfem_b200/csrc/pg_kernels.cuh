// pg_kernels.cuh -- the assembly kernels.
//
//   k_cut_elements   one warp per cut element: volumetric sub-element quadrature with enriched
//                    B-matrices plus the cohesive elements' traction-separation contributions
//                    (src/Assembler.cpp:223-365); writes the element matrix/vector to a scratch
//                    area, the trial internal variables and the damage zones.  FP64 throughout.
//   k_rows_fast      one thread per K row whose adjacent elements are all uncut: recomputes the
//                    element geometry of every adjacent element from node coordinates, keeps the
//                    row in registers (one accumulator per neighbour node) and writes each CSR
//                    value of the row exactly once, plus the residual entry.  No atomics; the
//                    summation order is the fixed adjacency order, so results are deterministic.
//   k_rows_slow      one thread per remaining row (rows touching cut elements, enrichment rows):
//                    same ownership, accumulates in place in the row's own CSR slots, taking the
//                    cut elements' rows from the scratch.
#pragma once

#include "pg_device.cuh"

namespace pgd {

// Geometry of an affine simplex (tri3 / tet4): physical gradients g[n][d] and the weight
// J * sum(W) of the reference's quadrature rule.  Jac(a,i) = sum_n dN_n/dr_a x_n[i]
// (Elem::transform_gradients); for the simplices that is x_{a+1} - x_0.
template <int DIM, typename T>
__device__ inline void simplex_geom(const T (*x)[DIM], T (*g)[DIM], T* J) {
  if (DIM == 2) {
    const T j00 = x[1][0] - x[0][0], j01 = x[1][1] - x[0][1];
    const T j10 = x[2][0] - x[0][0], j11 = x[2][1] - x[0][1];
    const T det = j00 * j11 - j01 * j10;
    const T s = T(1) / det;
    const T i00 = j11 * s, i11 = j00 * s, i01 = (T(-1) * j01) * s, i10 = (T(-1) * j10) * s;
    // dNdr = (-1,-1), (1,0), (0,1)
    g[0][0] = i00 * T(-1) + i01 * T(-1); g[0][1] = i10 * T(-1) + i11 * T(-1);
    g[1][0] = i00; g[1][1] = i10;
    g[2][0] = i01; g[2][1] = i11;
    *J = det;
  } else {
    T a[3][3];
    for (int r = 0; r < 3; ++r)
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
    for (int i = 0; i < 3; ++i) {
      g[0][i] = -(R[i][0] + R[i][1] + R[i][2]) * s;
      g[1][i] = R[i][0] * s; g[2][i] = R[i][1] * s; g[3][i] = R[i][2] * s;
    }
    *J = det;
  }
}

// sigma = D eps with the linear-elastic zero pattern (LinearElasticIsotropicMaterial::computeStress)
template <int DIM, typename T>
__device__ inline void lei_stress(const T* D, const T* e, T* s) {
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

// Weight sum of the reference rules for the uncut parents: tri3 order 3 and tet4 order 3.
__device__ __host__ inline double tri4_wsum() { return ((-0.28125 + 0.260416666666666666666666666666665) + 0.260416666666666666666666666666665) + 0.260416666666666666666666666666665; }
__device__ __host__ inline double tet5_wsum() { return (((-0.8 + 0.45) + 0.45) + 0.45) + 0.45; }

// Contribution of one uncut simplex element to row (local node la, dof q):
// kv[lb][q2] = wgt * (B_la^T D B_lb)[q][q2], rv = wgt * (B_la^T sigma)[q].
template <int DIM, typename T>
__device__ inline void simplex_row(const DevProblem& P, int e, int la, int q, const T* D, int (*nodes_out), T (*kv)[DIM], T* rv) {
  constexpr int NPE = DIM + 1;
  constexpr int NV = (DIM == 2) ? 3 : 6;
  T x[NPE][DIM], u[NPE][DIM], g[NPE][DIM], J;
#pragma unroll
  for (int n = 0; n < NPE; ++n) {
    const int nd = __ldg(&P.conn[(size_t)e * NPE + n]);
    nodes_out[n] = nd;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      if (sizeof(T) == 4) x[n][d] = (T)__ldg(&P.Xf[(size_t)nd * DIM + d]);
      else x[n][d] = (T)__ldg(&P.X[(size_t)nd * DIM + d]);
      u[n][d] = (T)__ldg(&P.U[(size_t)nd * DIM + d]);
    }
  }
  simplex_geom<DIM, T>(x, g, &J);
  const T wgt = J * (T)((DIM == 2) ? tri4_wsum() : tet5_wsum());
  // strain (Voigt, engineering shear) + macroscale strain
  T eps[NV];
  if (DIM == 2) {
    T e0 = 0, e1 = 0, e2 = 0;
#pragma unroll
    for (int n = 0; n < NPE; ++n) { e0 += g[n][0] * u[n][0]; e1 += g[n][1] * u[n][1]; e2 += g[n][1] * u[n][0] + g[n][0] * u[n][1]; }
    eps[0] = e0; eps[1] = e1; eps[2] = e2;
  } else {
    T e0 = 0, e1 = 0, e2 = 0, e3 = 0, e4 = 0, e5 = 0;
#pragma unroll
    for (int n = 0; n < NPE; ++n) {
      e0 += g[n][0] * u[n][0]; e1 += g[n][1] * u[n][1]; e2 += g[n][2] * u[n][2];
      e3 += g[n][2] * u[n][1] + g[n][1] * u[n][2];
      e4 += g[n][2] * u[n][0] + g[n][0] * u[n][2];
      e5 += g[n][1] * u[n][0] + g[n][0] * u[n][1];
    }
    eps[0] = e0; eps[1] = e1; eps[2] = e2; eps[3] = e3; eps[4] = e4; eps[5] = e5;
  }
  if (P.subscale) {
#pragma unroll
    for (int v = 0; v < NV; ++v) eps[v] += (T)P.eps_macro[v];
  }
  T sig[NV];
  lei_stress<DIM, T>(D, eps, sig);
  // t = B_la(:, q)^T D  (row of B^T D for local row la*DIM+q)
  T bq[NV], t[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) bq[v] = bmat<T>(DIM, v, q, g[la]);
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    T s = 0;
#pragma unroll
    for (int w = 0; w < NV; ++w) s += bq[w] * D[w * NV + v];
    t[v] = s;
  }
  T r = 0;
#pragma unroll
  for (int v = 0; v < NV; ++v) r += bq[v] * sig[v];
  *rv = wgt * r;
#pragma unroll
  for (int lb = 0; lb < NPE; ++lb) {
#pragma unroll
    for (int q2 = 0; q2 < DIM; ++q2) {
      T s = 0;
#pragma unroll
      for (int v = 0; v < NV; ++v) s += t[v] * bmat<T>(DIM, v, q2, g[lb]);
      kv[lb][q2] = wgt * s;
    }
  }
}

// Rows whose elements are all uncut simplices; MAXNB neighbour DOF nodes at most.
template <int DIM, int MAXNB, typename T>
__global__ void __launch_bounds__(128) k_rows_fast(DevProblem P) {
  constexpr int NPE = DIM + 1;
  constexpr int NV = (DIM == 2) ? 3 : 6;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= P.n_fast_rows) return;
  const int row = __ldg(&P.fast_rows[t]);
  const int a = row / DIM, q = row - a * DIM;
  const int na = __ldg(&P.dn_node[a]);
  const int gdof = __ldg(&P.node_dof[(size_t)na * DIM + q]);
  const int nb0 = __ldg(&P.dn_nbr_off[a]);
  const int nn = __ldg(&P.dn_nbr_off[a + 1]) - nb0;
  int nbr[MAXNB];
#pragma unroll
  for (int k = 0; k < MAXNB; ++k) nbr[k] = (k < nn) ? __ldg(&P.dn_nbr[nb0 + k]) : -1;
  // D of the two bulk materials in the arithmetic type
  T Dm[2][NV * NV];
#pragma unroll
  for (int m = 0; m < 2; ++m)
#pragma unroll
    for (int i = 0; i < NV; ++i)
#pragma unroll
      for (int j = 0; j < NV; ++j) Dm[m][i * NV + j] = (sizeof(T) == 4) ? (T)P.Df[m][i * NV + j] : (T)P.D[m][i * NV + j];
  double acc[MAXNB][DIM];
#pragma unroll
  for (int k = 0; k < MAXNB; ++k)
#pragma unroll
    for (int d = 0; d < DIM; ++d) acc[k][d] = 0.0;
  double racc = 0.0;
  const int ad0 = __ldg(&P.dn_adj_off[a]), ad1 = __ldg(&P.dn_adj_off[a + 1]);
  for (int s = ad0; s < ad1; ++s) {
    const int ent = __ldg(&P.dn_adj[s]);
    const int e = ent >> 5, la = ent & 31;
    const int m = __ldg(&P.emat[e]);
    int nodes[NPE];
    T kv[NPE][DIM], rv;
    simplex_row<DIM, T>(P, e, la, q, m ? Dm[1] : Dm[0], nodes, kv, &rv);
    racc += (double)rv;
#pragma unroll
    for (int lb = 0; lb < NPE; ++lb) {
      const int db = __ldg(&P.node_dn[nodes[lb]]);
#pragma unroll
      for (int k = 0; k < MAXNB; ++k)
        if (nbr[k] == db) {
#pragma unroll
          for (int d = 0; d < DIM; ++d) acc[k][d] += (double)kv[lb][d];
        }
    }
  }
  const bool rf = gdof < P.n_free;
  const int rr = rf ? gdof : gdof - P.n_free;
  const int bF = rf ? 0 : 2, bC = rf ? 1 : 3;
  if (P.flags & FLAG_JAC) {
    int pF = __ldg(&P.rp[bF][rr]), pC = __ldg(&P.rp[bC][rr]);
    double* vF = P.val[bF];
    double* vC = P.val[bC];
#pragma unroll
    for (int k = 0; k < MAXNB; ++k) {
      if (k < nn) {
        const int mask = __ldg(&P.dn_mask[nbr[k]]);
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
          if (mask & (1 << d)) vF[pF++] = acc[k][d];
          else vC[pC++] = acc[k][d];
        }
      }
    }
  }
  if (P.flags & FLAG_FUNC) {
    if (rf) P.Pf[rr] = racc; else P.Pp[rr] = racc;
  }
}

// Position of neighbour DOF node db in the sorted neighbour list of row node a.
__device__ inline int find_slot(const int* nbr, int n, int db) {
  int lo = 0, hi = n - 1;
  while (lo <= hi) {
    const int mid = (lo + hi) >> 1;
    const int v = __ldg(&nbr[mid]);
    if (v == db) return mid;
    if (v < db) lo = mid + 1; else hi = mid - 1;
  }
  return -1;
}

// All remaining rows: accumulate in the row's own CSR slots (the row belongs to this thread).
template <int DIM>
__global__ void __launch_bounds__(128) k_rows_slow(DevProblem P) {
  constexpr int NPE = DIM + 1;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= P.n_slow_rows) return;
  const int row = __ldg(&P.slow_rows[t]);
  const int a = row / DIM, q = row - a * DIM;
  const int na = __ldg(&P.dn_node[a]);
  const int gdof = __ldg(&P.node_dof[(size_t)na * DIM + q]);
  const int nb0 = __ldg(&P.dn_nbr_off[a]);
  const int nn = __ldg(&P.dn_nbr_off[a + 1]) - nb0;
  const bool rf = gdof < P.n_free;
  const int rr = rf ? gdof : gdof - P.n_free;
  const int bF = rf ? 0 : 2, bC = rf ? 1 : 3;
  const bool jac = (P.flags & FLAG_JAC) != 0;
  const int pF0 = __ldg(&P.rp[bF][rr]), pF1 = __ldg(&P.rp[bF][rr + 1]);
  const int pC0 = __ldg(&P.rp[bC][rr]), pC1 = __ldg(&P.rp[bC][rr + 1]);
  double* vF = P.val[bF];
  double* vC = P.val[bC];
  if (jac) {
    for (int p = pF0; p < pF1; ++p) vF[p] = 0.0;
    for (int p = pC0; p < pC1; ++p) vC[p] = 0.0;
  }
  double racc = 0.0;
  const int ad0 = __ldg(&P.dn_adj_off[a]), ad1 = __ldg(&P.dn_adj_off[a + 1]);
  for (int s = ad0; s < ad1; ++s) {
    const int ent = __ldg(&P.dn_adj[s]);
    const int e = ent >> 5, la = ent & 31;
    const int c = __ldg(&P.cut_of[e]);
    if (c < 0) {
      const int m = __ldg(&P.emat[e]);
      int nodes[NPE];
      double kv[NPE][DIM], rv;
      simplex_row<DIM, double>(P, e, la, q, P.D[m], nodes, kv, &rv);
      racc += rv;
      if (jac)
        for (int lb = 0; lb < NPE; ++lb) {
          const int db = __ldg(&P.node_dn[nodes[lb]]);
          const int k = find_slot(P.dn_nbr + nb0, nn, db);
          if (k < 0) { atomicOr(P.err, ERR_BAD_SLOT); continue; }
          const int mask = __ldg(&P.dn_mask[db]);
          int f = __ldg(&P.dn_nbr_pf[nb0 + k]), cc = __ldg(&P.dn_nbr_pc[nb0 + k]);
          for (int d = 0; d < DIM; ++d) {
            if (mask & (1 << d)) vF[pF0 + f++] += kv[lb][d];
            else vC[pC0 + cc++] += kv[lb][d];
          }
        }
    } else {
      const int o0 = __ldg(&P.cut_node_off[c]);
      const int mn = __ldg(&P.cut_node_off[c + 1]) - o0;
      const int nd = mn * DIM;
      const double* kr = P.ke + __ldg(&P.ke_off[c]) + (size_t)(la * DIM + q) * nd;
      racc += P.re[__ldg(&P.re_off[c]) + la * DIM + q];
      if (jac)
        for (int lb = 0; lb < mn; ++lb) {
          const int db = __ldg(&P.node_dn[__ldg(&P.cut_nodes[o0 + lb])]);
          const int k = find_slot(P.dn_nbr + nb0, nn, db);
          if (k < 0) { atomicOr(P.err, ERR_BAD_SLOT); continue; }
          const int mask = __ldg(&P.dn_mask[db]);
          int f = __ldg(&P.dn_nbr_pf[nb0 + k]), cc = __ldg(&P.dn_nbr_pc[nb0 + k]);
          for (int d = 0; d < DIM; ++d) {
            if (mask & (1 << d)) vF[pF0 + f++] += kr[lb * DIM + d];
            else vC[pC0 + cc++] += kr[lb * DIM + d];
          }
        }
    }
  }
  if (P.flags & FLAG_FUNC) {
    if (rf) P.Pf[rr] = racc; else P.Pp[rr] = racc;
  }
}

// Doubles of shared memory one warp of k_cut_elements uses for elements of up to md DOFs.
__host__ __device__ inline int cut_smem_per_warp(int md, int nv) { return 2 * md * md + md * nv + 4 * md + 2 * nv + 40; }

// One warp per cut element.  Shared memory per warp: Ke (nd x nd), BtD (nd x NV), Re (nd),
// U (nd), gradients (mn x DIM), strain/stress, cohesive block (up to (2*nh*DIM)^2).
template <int DIM>
__global__ void __launch_bounds__(128) k_cut_elements(DevProblem P, int max_nd) {
  constexpr int NV = (DIM == 2) ? 3 : 6;
  extern __shared__ double smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wpb = blockDim.x >> 5;
  const int c = blockIdx.x * wpb + warp;
  const int per_warp = cut_smem_per_warp(max_nd, NV);
  double* Ke = smem + (size_t)warp * per_warp;
  double* BtD = Ke + max_nd * max_nd;
  double* Re = BtD + max_nd * NV;
  double* Ul = Re + max_nd;
  double* G = Ul + max_nd;        // mn * DIM gradients of the current qp
  double* es = G + max_nd;        // eps (NV), sigma (NV)
  double* Kc = es + 2 * NV;       // cohesive block
  double* cw = Kc + max_nd * max_nd + max_nd;  // cohesive scalars: delta, T, Dm, RDR, tracR
  if (c >= P.ncut) return;
  const int o0 = P.cut_node_off[c];
  const int mn = P.cut_node_off[c + 1] - o0;
  const int nd = mn * DIM;
  for (int i = lane; i < nd * nd; i += 32) Ke[i] = 0.0;
  for (int i = lane; i < nd; i += 32) {
    Re[i] = 0.0;
    const int node = P.cut_nodes[o0 + i / DIM];
    Ul[i] = P.U[(size_t)node * DIM + (i % DIM)];
  }
  __syncwarp();
  const int q0 = P.cut_qp_off[c], q1 = P.cut_qp_off[c + 1];
  for (int qp = q0; qp < q1; ++qp) {
    const double wgt = P.qp_wgt[qp];
    const double* D = P.D[P.qp_mat[qp]];
    const double* gsrc = P.qp_grad + P.qp_grad_off[qp];
    for (int i = lane; i < nd; i += 32) G[i] = gsrc[i];
    __syncwarp();
    // eps = B U (+ eps_macro), sigma = D eps
    if (lane < NV) {
      double s = 0.0;
      for (int k = 0; k < nd; ++k) s += bmat<double>(DIM, lane, k % DIM, G + (k / DIM) * DIM) * Ul[k];
      if (P.subscale) s += P.eps_macro[lane];
      es[lane] = s;
    }
    __syncwarp();
    if (lane == 0) lei_stress<DIM, double>(D, es, es + NV);
    // BtD(i, v) = sum_w B(w, i) D(w, v)
    for (int idx = lane; idx < nd * NV; idx += 32) {
      const int i = idx / NV, v = idx - i * NV;
      double s = 0.0;
      for (int w = 0; w < NV; ++w) s += bmat<double>(DIM, w, i % DIM, G + (i / DIM) * DIM) * D[w * NV + v];
      BtD[idx] = s;
    }
    __syncwarp();
    for (int idx = lane; idx < nd * nd; idx += 32) {
      const int i = idx / nd, j = idx - i * nd;
      double s = 0.0;
      for (int v = 0; v < NV; ++v) s += BtD[i * NV + v] * bmat<double>(DIM, v, j % DIM, G + (j / DIM) * DIM);
      Ke[idx] += wgt * s;
    }
    for (int i = lane; i < nd; i += 32) {
      double s = 0.0;
      for (int v = 0; v < NV; ++v) s += bmat<double>(DIM, v, i % DIM, G + (i / DIM) * DIM) * es[NV + v];
      Re[i] += wgt * s;
    }
    __syncwarp();
  }
  // cohesive elements
  const int ce0 = P.cut_coh_off[c], ce1 = P.cut_coh_off[c + 1];
  for (int ce = ce0; ce < ce1; ++ce) {
    const int nh = P.coh_nh[ce];
    const int* cl = P.coh_local + P.coh_local_off[ce];
    const int ncd = 2 * nh * DIM;
    for (int i = lane; i < ncd * ncd + ncd; i += 32) Kc[i] = 0.0;  // Kc then Pc
    __syncwarp();
    double* Pc = Kc + ncd * ncd;
    const int cq0 = P.coh_qp_off[ce], cq1 = P.coh_qp_off[ce + 1];
    for (int cq = cq0; cq < cq1; ++cq) {
      const double* N = P.cqp_N + (size_t)cq * nh;
      const double* R = P.cqp_R + (size_t)cq * DIM * DIM;
      double* dl = cw;            // DIM
      double* T = cw + 4;         // DIM
      double* Dc = cw + 8;        // DIM*DIM
      double* RDR = cw + 20;      // DIM*DIM
      double* tR = cw + 30;       // DIM
      if (lane == 0) {
        double d0[3] = {0, 0, 0};
        for (int d = 0; d < DIM; ++d)
          for (int n = 0; n < nh; ++n) d0[d] += N[n] * (Ul[cl[n + nh] * DIM + d] - Ul[cl[n] * DIM + d]);
        for (int i = 0; i < DIM; ++i) {
          double s = 0.0;
          for (int j = 0; j < DIM; ++j) s += R[i * DIM + j] * d0[j];
          dl[i] = s;
        }
        const int iv = P.cqp_isv[cq];
        double isv[2] = {0.0, 0.0};
        for (int v = 0; v < P.coh.nvar; ++v) isv[v] = P.isv_committed[iv + v];
        uint8_t z;
        coh_law(P.coh, DIM, dl, T, Dc, isv, &z);
        for (int v = 0; v < P.coh.nvar; ++v) P.isv_trial[iv + v] = isv[v];
        P.zone[cq] = z;
        // RDR = (R^T D) R ; tracR = R^T T
        double RtD[9];
        for (int i = 0; i < DIM; ++i)
          for (int k = 0; k < DIM; ++k) {
            double s = 0.0;
            for (int j = 0; j < DIM; ++j) s += R[j * DIM + i] * Dc[j * DIM + k];
            RtD[i * DIM + k] = s;
          }
        for (int i = 0; i < DIM; ++i)
          for (int l = 0; l < DIM; ++l) {
            double s = 0.0;
            for (int k = 0; k < DIM; ++k) s += RtD[i * DIM + k] * R[k * DIM + l];
            RDR[i * DIM + l] = s;
          }
        for (int i = 0; i < DIM; ++i) {
          double s = 0.0;
          for (int j = 0; j < DIM; ++j) s += R[j * DIM + i] * T[j];
          tR[i] = s;
        }
      }
      __syncwarp();
      const double w = P.cqp_wgt[cq];
      for (int idx = lane; idx < ncd * ncd; idx += 32) {
        const int r = idx / ncd, col = idx - r * ncd;
        const int n1 = r / DIM, d1 = r - n1 * DIM, n2 = col / DIM, d2 = col - n2 * DIM;
        const int a1 = n1 % nh, a2 = n2 % nh;
        const double val = N[a1] * N[a2] * RDR[d1 * DIM + d2];
        const double sgn = ((n1 >= nh) == (n2 >= nh)) ? 1.0 : -1.0;
        Kc[idx] += w * (sgn * val);
      }
      for (int idx = lane; idx < ncd; idx += 32) {
        const int n = idx / DIM, d = idx - n * DIM;
        const double val = N[n % nh] * tR[d];
        Pc[idx] += w * ((n >= nh) ? val : -val);
      }
      __syncwarp();
    }
    // add the cohesive block into the element matrix through the cohesive node map
    for (int idx = lane; idx < ncd * ncd; idx += 32) {
      const int r = idx / ncd, col = idx - r * ncd;
      const int rd = cl[r / DIM] * DIM + (r % DIM), cd = cl[col / DIM] * DIM + (col % DIM);
      Ke[rd * nd + cd] += Kc[idx];
    }
    __syncwarp();
    if (lane == 0)
      for (int r = 0; r < ncd; ++r) Re[cl[r / DIM] * DIM + (r % DIM)] += Pc[r];
    __syncwarp();
  }
  double* ko = P.ke + P.ke_off[c];
  double* ro = P.re + P.re_off[c];
  bool bad = false;
  for (int i = lane; i < nd * nd; i += 32) { ko[i] = Ke[i]; bad |= !isfinite(Ke[i]); }
  for (int i = lane; i < nd; i += 32) { ro[i] = Re[i]; bad |= !isfinite(Re[i]); }
  if (bad) atomicOr(P.err, ERR_NONFINITE);
}

}  // namespace pgd
