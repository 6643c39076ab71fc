// pg_stencil.cuh -- structured-grid fast path of the row assembly.
//
// The background meshes are the reference's structured grids (Mesh::generate_mesh,
// src/Mesh.cpp:386-604): quads split into two tri3 with the union-jack alternation, hexes split
// into six tet4.  Away from the domain boundary and from cut elements every DOF node of such a
// grid has the same neighbourhood up to its class (the parity of i + j for tri3, a single class
// for tet4).  The tables below give, for each class, the neighbour offsets in row order and, for
// each adjacent element, its cell offset, its index within the cell, the row node's local index
// and the neighbour slot of each of its nodes.  They restate the reference's cell-splitting
// tables in row-owner form; the set-up checks every node it sends here against them and sends
// any node that does not match to the general kernel.  With the slots known at compile time the
// whole block row lives in registers, node and element ids come from grid arithmetic (no
// adjacency or connectivity reads) and each row is written with contiguous stores.
#pragma once

#include "pg_kernels.cuh"

namespace pgd {

struct Tri3Stencil0 {
  static constexpr int NN = 9, NADJ = 8;
  // neighbour offsets (di, dj, dk) in row (node id) order
  __host__ __device__ static constexpr int off(int s, int d) {
    constexpr int t[NN][3] = {{-1, -1, 0}, {0, -1, 0}, {1, -1, 0}, {-1, 0, 0}, {0, 0, 0}, {1, 0, 0}, {-1, 1, 0}, {0, 1, 0}, {1, 1, 0}};
    return t[s][d];
  }
  // adjacent elements: cell offset (di, dj, dk), element within the cell, local index of the
  // row node, neighbour slot of each element node in connectivity order
  __host__ __device__ static constexpr int ent(int a, int c) {
    constexpr int t[NADJ][8] = {{-1, -1, 0, 0, 2, 0, 1, 4}, {-1, -1, 0, 1, 1, 0, 4, 3}, {0, -1, 0, 0, 2, 1, 2, 4}, {0, -1, 0, 1, 2, 2, 5, 4}, {-1, 0, 0, 0, 1, 3, 4, 6}, {-1, 0, 0, 1, 0, 4, 7, 6}, {0, 0, 0, 0, 0, 4, 5, 8}, {0, 0, 0, 1, 0, 4, 8, 7}};
    return t[a][c];
  }
};
struct Tri3Stencil1 {
  static constexpr int NN = 5, NADJ = 4;
  // neighbour offsets (di, dj, dk) in row (node id) order
  __host__ __device__ static constexpr int off(int s, int d) {
    constexpr int t[NN][3] = {{0, -1, 0}, {-1, 0, 0}, {0, 0, 0}, {1, 0, 0}, {0, 1, 0}};
    return t[s][d];
  }
  // adjacent elements: cell offset (di, dj, dk), element within the cell, local index of the
  // row node, neighbour slot of each element node in connectivity order
  __host__ __device__ static constexpr int ent(int a, int c) {
    constexpr int t[NADJ][8] = {{-1, -1, 0, 1, 1, 0, 2, 1}, {0, -1, 0, 1, 2, 0, 3, 2}, {-1, 0, 0, 0, 1, 1, 2, 4}, {0, 0, 0, 0, 0, 2, 3, 4}};
    return t[a][c];
  }
};
struct Tet4Stencil0 {
  static constexpr int NN = 15, NADJ = 24;
  // neighbour offsets (di, dj, dk) in row (node id) order
  __host__ __device__ static constexpr int off(int s, int d) {
    constexpr int t[NN][3] = {{-1, -1, -1}, {0, -1, -1}, {-1, 0, -1}, {0, 0, -1}, {-1, -1, 0}, {0, -1, 0}, {-1, 0, 0}, {0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {1, 1, 0}, {0, 0, 1}, {1, 0, 1}, {0, 1, 1}, {1, 1, 1}};
    return t[s][d];
  }
  // adjacent elements: cell offset (di, dj, dk), element within the cell, local index of the
  // row node, neighbour slot of each element node in connectivity order
  __host__ __device__ static constexpr int ent(int a, int c) {
    constexpr int t[NADJ][9] = {{-1, -1, -1, 0, 3, 0, 3, 2, 7}, {-1, -1, -1, 1, 3, 0, 2, 6, 7}, {-1, -1, -1, 2, 3, 0, 6, 4, 7}, {-1, -1, -1, 3, 2, 0, 5, 7, 4}, {-1, -1, -1, 4, 2, 1, 5, 7, 0}, {-1, -1, -1, 5, 1, 1, 7, 3, 0}, {0, -1, -1, 1, 2, 1, 3, 7, 8}, {0, -1, -1, 2, 1, 1, 7, 5, 8}, {-1, 0, -1, 3, 1, 2, 7, 9, 6}, {-1, 0, -1, 4, 1, 3, 7, 9, 2}, {0, 0, -1, 2, 2, 3, 9, 7, 10}, {0, 0, -1, 3, 3, 3, 8, 10, 7}, {-1, -1, 0, 0, 1, 4, 7, 6, 11}, {-1, -1, 0, 5, 2, 5, 11, 7, 4}, {0, -1, 0, 0, 2, 5, 8, 7, 12}, {0, -1, 0, 1, 1, 5, 7, 11, 12}, {-1, 0, 0, 4, 0, 7, 11, 13, 6}, {-1, 0, 0, 5, 0, 7, 13, 9, 6}, {0, 0, 0, 0, 0, 7, 10, 9, 14}, {0, 0, 0, 1, 0, 7, 9, 13, 14}, {0, 0, 0, 2, 0, 7, 13, 11, 14}, {0, 0, 0, 3, 0, 7, 12, 14, 11}, {0, 0, 0, 4, 3, 8, 12, 14, 7}, {0, 0, 0, 5, 3, 8, 14, 10, 7}};
    return t[a][c];
  }
};


struct GridInfo {
  int nx, ny, nz;
};

// sigma = D eps for the isotropic linear-elastic D (only its nonzero entries)
template <int DIM, typename T>
__device__ __forceinline__ void lei_stress_iso(const T* d, const T* e, T* s) {
  // d: 2D {D00, D01, D10, D11, D22}; 3D {D00, D01, D02, D10, D11, D12, D20, D21, D22, D33, D44, D55}
  if (DIM == 2) { s[0] = d[0] * e[0] + d[1] * e[1]; s[1] = d[2] * e[0] + d[3] * e[1]; s[2] = d[4] * e[2]; }
  else {
    s[0] = d[0] * e[0] + d[1] * e[1] + d[2] * e[2];
    s[1] = d[3] * e[0] + d[4] * e[1] + d[5] * e[2];
    s[2] = d[6] * e[0] + d[7] * e[1] + d[8] * e[2];
    s[3] = d[9] * e[3]; s[4] = d[10] * e[4]; s[5] = d[11] * e[5];
  }
}
// part = (B_a(:, q))^T D using only the nonzero entries of the isotropic D (the zero terms of the
// reference's SmallStrainKFast contribute exact zeros).
template <int DIM, typename T>
__device__ __forceinline__ void part_iso(const T* d, const T* ga, int q, T* part) {
  if (DIM == 2) {
    if (q == 0) { part[0] = ga[0] * d[0]; part[1] = ga[0] * d[1]; part[2] = ga[1] * d[4]; }
    else        { part[0] = ga[1] * d[2]; part[1] = ga[1] * d[3]; part[2] = ga[0] * d[4]; }
  } else {
    if (q == 0) { part[0] = ga[0] * d[0]; part[1] = ga[0] * d[1]; part[2] = ga[0] * d[2]; part[3] = T(0); part[4] = ga[2] * d[10]; part[5] = ga[1] * d[11]; }
    else if (q == 1) { part[0] = ga[1] * d[3]; part[1] = ga[1] * d[4]; part[2] = ga[1] * d[5]; part[3] = ga[2] * d[9]; part[4] = T(0); part[5] = ga[0] * d[11]; }
    else { part[0] = ga[2] * d[6]; part[1] = ga[2] * d[7]; part[2] = ga[2] * d[8]; part[3] = ga[1] * d[9]; part[4] = ga[0] * d[10]; part[5] = T(0); }
  }
}

// the nonzero entries of an isotropic D (36 entries, row-major) in lei_stress_iso's order
template <int DIM, typename T>
__device__ __forceinline__ void iso_from(const T* D, T* d) {
  constexpr int n = (DIM == 2) ? 5 : 12;
  constexpr int i2[5] = {0, 1, 3, 4, 8};
  constexpr int i3[12] = {0, 1, 2, 6, 7, 8, 12, 13, 14, 21, 28, 35};
#pragma unroll
  for (int k = 0; k < n; ++k) d[k] = D[(DIM == 2) ? i2[k] : i3[k]];
}

template <int DIM, typename T>
__device__ __forceinline__ void iso_d(const DevProblem& P, int m, T* d) {
  const int* idx;
  constexpr int n = (DIM == 2) ? 5 : 12;
  const int i2[5] = {0, 1, 3, 4, 8};
  const int i3[12] = {0, 1, 2, 6, 7, 8, 12, 13, 14, 21, 28, 35};
#pragma unroll
  for (int k = 0; k < n; ++k) {
    const int o = (DIM == 2) ? i2[k] : i3[k];
    d[k] = (sizeof(T) == 4) ? (T)__ldg(&P.Dfd[m * 36 + o]) : (T)__ldg(&P.Dd[m * 36 + o]);
  }
  (void)idx;
}

// The last adjacent element (in adjacency order) that has neighbour slot s among its nodes.
template <class S, int NPE>
__host__ __device__ constexpr int slot_last_touch(int s) {
  int l = -1;
  for (int a = 0; a < S::NADJ; ++a)
    for (int n = 0; n < NPE; ++n)
      if (S::ent(a, 5 + n) == s) l = a;
  return l;
}

// Rows of one stencil node.  Q < 0: all dim rows in one thread; Q >= 0: row Q only.  JAC = false
// compiles the residual alone (no stiffness accumulators, no CSR writes).  Each neighbour block is
// stored as soon as the last element touching it has been added (the slots are compile-time, so
// the store points are too): its registers are free for the rest of the walk.
template <class S, int DIM, typename T, int Q, bool JAC = true>
__device__ __forceinline__ void stencil_rows(const DevProblem& P, const GridInfo& gi, int nid, int g0, int row0,
                                             double* stage = nullptr) {
  constexpr int NPE = DIM + 1;
  constexpr int NV = (DIM == 2) ? 3 : 6;
  constexpr int ND = (DIM == 2) ? 5 : 12;
  constexpr int QB = (Q < 0) ? 0 : Q, QE = (Q < 0) ? DIM : Q + 1;
  const int sx = gi.nx + 1, sxy = sx * (gi.ny + 1);
  const int i = nid % sx, j = (nid / sx) % (gi.ny + 1), k = nid / sxy;
  const bool jac = JAC && (P.flags & FLAG_JAC) != 0;  // uniform over the launch
  double acc[JAC ? S::NN : 1][QE - QB][DIM];
  if constexpr (JAC) {
#pragma unroll
    for (int s = 0; s < S::NN; ++s)
#pragma unroll
      for (int q = 0; q < QE - QB; ++q)
#pragma unroll
        for (int d = 0; d < DIM; ++d) acc[s][q][d] = 0.0;
  }
  double r[QE - QB];
#pragma unroll
  for (int q = 0; q < QE - QB; ++q) r[q] = 0.0;
#pragma unroll
  for (int a = 0; a < S::NADJ; ++a) {
    const int ci = i + S::ent(a, 0), cj = j + S::ent(a, 1), ck = k + S::ent(a, 2);
    const int e = (DIM == 2) ? 2 * (cj * gi.nx + ci) + S::ent(a, 3) : 6 * ((ck * gi.ny + cj) * gi.nx + ci) + S::ent(a, 3);
    const int m = __ldg(&P.emat[e]);
    double x[NPE][DIM], u[NPE][DIM], g[NPE][DIM], J;
#pragma unroll
    for (int n = 0; n < NPE; ++n) {
      const int sl = S::ent(a, 5 + n);
      const int id = nid + S::off(sl, 0) + S::off(sl, 1) * sx + S::off(sl, 2) * sxy;
      load_node<DIM>(P.X, id, x[n]);
      load_node<DIM>(P.U, id, u[n]);
    }
    // geometry, strain, stress and the internal force in FP64 (the Newton residual)
    simplex_geom<DIM, double>(x, g, &J);
    const double w = J * ((DIM == 2) ? tri4_wsum() : tet5_wsum());
    double eps[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) eps[v] = 0;
#pragma unroll
    for (int n = 0; n < NPE; ++n) add_strain<DIM, double>(g[n], u[n], eps);
    if (P.subscale) {
#pragma unroll
      for (int v = 0; v < NV; ++v) eps[v] += P.eps_macro[v];
    }
    // D of the element's material from the descriptor (kernel parameter space), per element:
    // keeping both materials' D in registers costs more registers than the loads
    double d[ND];
    iso_from<DIM, double>(P.D[m], d);
    double sig[NV];
    lei_stress_iso<DIM, double>(d, eps, sig);
    const int la = S::ent(a, 4);
    // the stiffness block products in T (FP32 in the mixed path), accumulated in FP64
    T gk[NPE][DIM];
#pragma unroll
    for (int n = 0; n < NPE; ++n)
#pragma unroll
      for (int dd = 0; dd < DIM; ++dd) gk[n][dd] = (T)g[n][dd];
    const T wk = (T)w;
    T dkv[ND];   // the tangent's D in the element-stiffness precision
    if constexpr (sizeof(T) == sizeof(double)) {
#pragma unroll
      for (int k2 = 0; k2 < ND; ++k2) dkv[k2] = (T)d[k2];
    } else {
      iso_from<DIM, T>(P.Df[m], dkv);
    }
    const T* dk = dkv;
#pragma unroll
    for (int q = QB; q < QE; ++q) {
      r[q - QB] += w * bt_sig<DIM, double>(g[la], sig, q);
      if constexpr (JAC) if (jac) {
        T part[NV];
        part_iso<DIM, T>(dk, gk[la], q, part);
#pragma unroll
        for (int lb = 0; lb < NPE; ++lb)
#pragma unroll
          for (int q2 = 0; q2 < DIM; ++q2) acc[S::ent(a, 5 + lb)][q - QB][q2] += (double)(wk * part_b<DIM, T>(part, gk[lb], q2));
      }
    }
    if constexpr (JAC) if (jac) {
      // the blocks no later element touches: to the caller's stage when it has one, else
      // straight to the CSR (a node's rows are consecutive, NN x DIM values each)
#pragma unroll
      for (int s = 0; s < S::NN; ++s) {
        if (slot_last_touch<S, NPE>(s) != a) continue;
#pragma unroll
        for (int q = QB; q < QE; ++q) {
          double* v = stage ? stage + (size_t)q * S::NN * DIM : P.val[0] + row0 + (size_t)q * S::NN * DIM;
#pragma unroll
          for (int d = 0; d < DIM; ++d) v[s * DIM + d] = acc[s][q - QB][d];
        }
      }
    }
  }
#pragma unroll
  for (int q = QB; q < QE; ++q)
    if (P.flags & FLAG_FUNC) P.Pf[g0 + q] = r[q - QB];
}

// 2D rows of the stencil node of this lane, staged: the lane's two rows (2 x NN x 2 values, one
// contiguous run of the CSR since a node's rows follow each other) go to the warp's shared-memory
// stage, then the warp writes the 32 runs with consecutive lanes on consecutive addresses, so a
// store instruction touches a few sectors instead of one per lane.  Every lane of the warp calls it
// (valid = false for padding entries); the warp's entries share one class.
constexpr int kStageStride = 37;   // doubles per lane in the stage (>= the longest run, 36; odd)
__host__ __device__ inline size_t stencil_stage_bytes(int threads) { return (size_t)threads * kStageStride * sizeof(double); }

template <class S, typename T>
__device__ __forceinline__ void stencil_rows_staged(const DevProblem& P, const GridInfo& gi, int4 v, bool valid,
                                                    double* stage) {
  constexpr int RUN = 2 * S::NN * 2;
  const int lane = threadIdx.x & 31;
  double* my = stage + (size_t)(threadIdx.x & ~31) * kStageStride;
  if (valid) stencil_rows<S, 2, T, -1>(P, gi, v.x, v.y, v.z, my + lane * kStageStride);
  if (!(P.flags & FLAG_JAC)) return;
  __syncwarp();
  const unsigned ok = __ballot_sync(0xffffffffu, valid);
  double* out = P.val[0];
  for (int i = lane; i < 32 * RUN; i += 32) {
    const int k = i / RUN, o = i - k * RUN;
    const int r0 = __shfl_sync(0xffffffffu, v.z, k);
    if ((ok >> k) & 1u) out[(size_t)r0 + o] = my[k * kStageStride + o];
  }
  __syncwarp();
}

// One thread per stencil node (2D) or per (stencil node, row) (3D, rows interleaved by warp so the
// row is warp-uniform).  st: {node id, first free DOF, first CSR slot of its first row, class} per
// node, class-sorted, each class padded to whole warps with node -1.  2D launches carry
// stencil_stage_bytes(blockDim.x) of dynamic shared memory.  JAC = false (residual only): one
// thread per stencil node in 2D and 3D, no shared memory.
template <int DIM, typename T, bool JAC = true>
__global__ void __launch_bounds__(128) k_rows_stencil(DevProblem P, GridInfo gi, const int4* __restrict__ st, int n) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if constexpr (!JAC) {
    if (t >= n) return;
    const int4 v = __ldg(&st[t]);
    if (v.x < 0) return;   // padding entry
    if constexpr (DIM == 2) {
      if (v.w == 0) stencil_rows<Tri3Stencil0, 2, double, -1, false>(P, gi, v.x, v.y, v.z);
      else stencil_rows<Tri3Stencil1, 2, double, -1, false>(P, gi, v.x, v.y, v.z);
    } else {
      stencil_rows<Tet4Stencil0, 3, double, -1, false>(P, gi, v.x, v.y, v.z);
    }
    return;
  }
  if (DIM == 2) {
    extern __shared__ double stage[];
    if (t - (int)(threadIdx.x & 31) >= n) return;   // whole warps only: n is a multiple of 32
    const int4 v = __ldg(&st[t]);
    if (v.w == 0) stencil_rows_staged<Tri3Stencil0, T>(P, gi, v, v.x >= 0, stage);
    else stencil_rows_staged<Tri3Stencil1, T>(P, gi, v, v.x >= 0, stage);
  } else {
    // a warp takes one row (q) of 32 consecutive stencil nodes, so q is uniform within a warp
    const int w = t >> 5, lane = t & 31;
    const int q = w % 3, node = (w / 3) * 32 + lane;
    if (node >= n) return;
    const int4 v = __ldg(&st[node]);
    if (v.x < 0) return;   // padding entry
    if (q == 0) stencil_rows<Tet4Stencil0, 3, T, 0>(P, gi, v.x, v.y, v.z);
    else if (q == 1) stencil_rows<Tet4Stencil0, 3, T, 1>(P, gi, v.x, v.y, v.z);
    else stencil_rows<Tet4Stencil0, 3, T, 2>(P, gi, v.x, v.y, v.z);
  }
}

// Residuals of one stencil node (all its rows) for the P.n_cases macroscale strains of a
// multi-strain pass: per adjacent element the geometry and the strain of U are formed once, then
// each case adds its strain and forms its stress and B^T sigma -- for each case the operations of
// stencil_rows with that case as eps_macro.
template <class S, int DIM>
__device__ __forceinline__ void stencil_resid_cases(const DevProblem& P, const GridInfo& gi, int nid, int g0) {
  constexpr int NPE = DIM + 1;
  constexpr int NV = (DIM == 2) ? 3 : 6;
  constexpr int ND = (DIM == 2) ? 5 : 12;
  constexpr int MC = 6;
  const int nc = P.n_cases;
  const int sx = gi.nx + 1, sxy = sx * (gi.ny + 1);
  const int i = nid % sx, j = (nid / sx) % (gi.ny + 1), k = nid / sxy;
  double r[MC][DIM];
#pragma unroll
  for (int c = 0; c < MC; ++c)
#pragma unroll
    for (int q = 0; q < DIM; ++q) r[c][q] = 0.0;
#pragma unroll
  for (int a = 0; a < S::NADJ; ++a) {
    const int ci = i + S::ent(a, 0), cj = j + S::ent(a, 1), ck = k + S::ent(a, 2);
    const int e = (DIM == 2) ? 2 * (cj * gi.nx + ci) + S::ent(a, 3) : 6 * ((ck * gi.ny + cj) * gi.nx + ci) + S::ent(a, 3);
    const int m = __ldg(&P.emat[e]);
    double x[NPE][DIM], u[NPE][DIM], g[NPE][DIM], J;
#pragma unroll
    for (int n = 0; n < NPE; ++n) {
      const int sl = S::ent(a, 5 + n);
      const int id = nid + S::off(sl, 0) + S::off(sl, 1) * sx + S::off(sl, 2) * sxy;
      load_node<DIM>(P.X, id, x[n]);
      load_node<DIM>(P.U, id, u[n]);
    }
    simplex_geom<DIM, double>(x, g, &J);
    const double w = J * ((DIM == 2) ? tri4_wsum() : tet5_wsum());
    double eps[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) eps[v] = 0;
#pragma unroll
    for (int n = 0; n < NPE; ++n) add_strain<DIM, double>(g[n], u[n], eps);
    double d[ND];
    iso_from<DIM, double>(P.D[m], d);
    const int la = S::ent(a, 4);
    double ga[DIM];
#pragma unroll
    for (int dd = 0; dd < DIM; ++dd) ga[dd] = g[0][dd];
#pragma unroll
    for (int n = 1; n < NPE; ++n)
      if (la == n)
#pragma unroll
        for (int dd = 0; dd < DIM; ++dd) ga[dd] = g[n][dd];
#pragma unroll
    for (int c = 0; c < MC; ++c) {
      if (c >= nc) break;
      double ek[NV], sig[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) ek[v] = eps[v] + P.eps_cases[c][v];
      lei_stress_iso<DIM, double>(d, ek, sig);
#pragma unroll
      for (int q = 0; q < DIM; ++q) r[c][q] += w * bt_sig<DIM, double>(ga, sig, q);
    }
  }
#pragma unroll
  for (int c = 0; c < MC; ++c) {
    if (c >= nc) break;
#pragma unroll
    for (int q = 0; q < DIM; ++q) P.Pf_cases[(size_t)c * P.n_free + g0 + q] = r[c][q];
  }
}

// One thread per stencil node: residuals of P.n_cases macroscale strains.
template <int DIM>
__global__ void __launch_bounds__(128) k_rows_stencil_cases(DevProblem P, GridInfo gi, const int4* __restrict__ st, int n) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int4 v = __ldg(&st[t]);
  if (v.x < 0) return;   // padding entry
  if constexpr (DIM == 2) {
    if (v.w == 0) stencil_resid_cases<Tri3Stencil0, 2>(P, gi, v.x, v.y);
    else stencil_resid_cases<Tri3Stencil1, 2>(P, gi, v.x, v.y);
  } else {
    stencil_resid_cases<Tet4Stencil0, 3>(P, gi, v.x, v.y);
  }
}

// Host-side copies of the tables for the set-up's check.
struct StencilView {
  int nn, nadj, npe;
  const int (*off)[3];
  const int* ent;  // nadj x (5 + npe)
};

}  // namespace pgd
