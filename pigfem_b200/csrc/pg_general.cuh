// pg_general.cuh -- block-parallel general rows (tri3 / tet4 meshes).
//
// The general rows are the DOF nodes the structured tiles do not take: boundary rows, nodes of
// cut elements and enrichment nodes.  Every bulk law is linear elastic, so the volumetric part of
// their rows does not depend on the state: the set-up sums each general node's cut and uncut
// elements' blocks into a static image (one DIM x DIM block per (node, neighbour slot),
// k_general_static) and its macroscale-strain response.  An assembly forms, from loads that are
// all independent of one another (the set-up flattened every index):
//   gen_block    one thread per (general node, neighbour slot) block: the static block plus the
//                cohesive blocks of the cohesive elements holding both nodes (kcoh, from the
//                cohesive pass) in adjacency order, then the block's CSR values, each written once;
//   gen_resid    a group of 8 lanes per general node: the static blocks times the displacements
//                (slot order), the macroscale-strain response and the cohesive tractions
//                (adjacency order), terms formed in parallel and summed in that order by shuffles.
// Every value is a sum in a fixed order, so results are bit-reproducible, and a residual-only
// assembly forms bitwise the residual of the full one.  An assembly launches two kernels:
// k_gen_first (the cohesive elements) and k_gen_rows (residuals and blocks).
#pragma once

#include "pg_stencil.cuh"

namespace pgd {

// Programmatic dependent launch: k_gen_rows may start while the kernel before it in the stream
// (k_gen_first in 2D, the tiles in 3D) still runs; griddepcontrol.wait returns once that grid has
// completed and its writes are visible (at once when the launch had no such dependency), so the
// cohesive blocks and tractions read after it are complete.  Threads that read none of them
// (nodes on no cohesive element) do not wait: their writes go to rows that kernel never touches.
__device__ __forceinline__ void dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
// Lets the dependent grid launch now (its blocks then do their independent loads).
__device__ __forceinline__ void dep_launch() { asm volatile("griddepcontrol.launch_dependents;" :::); }

template <int DIM>
__device__ __forceinline__ void gen_block(const DevProblem& P, int b) {
  constexpr int D2 = DIM * DIM;
  const int4 bd = __ldg(&P.gblk[b]);
  const int cl0 = __ldg(&P.gblk_cl[b]), cl1 = __ldg(&P.gblk_cl[b + 1]);
  const int node = bd.x, slot = bd.y;
  // the destination of the block's values depends on the descriptor alone: its loads are issued
  // before the sums, so they overlap the loads of the terms
  const int4 gd = __ldg(&P.gdesc[node]);
  const int mk = __ldg(&P.dn_nbr_mask[gd.z + slot]);
  const int pre = __ldg(&P.nbr_pre[gd.z + slot]);
  const int* rd = P.growd + (size_t)node * 3 * DIM;
  int rrow[DIM], rF[DIM], rC[DIM];
#pragma unroll
  for (int q = 0; q < DIM; ++q) { rrow[q] = __ldg(&rd[q]); rF[q] = __ldg(&rd[DIM + q]); rC[q] = __ldg(&rd[2 * DIM + q]); }
  double acc[D2];
  const double* S = P.stat + (size_t)bd.z * D2;
#pragma unroll
  for (int i = 0; i < D2; ++i) acc[i] = __ldg(&S[i]);
  // the cohesive blocks below come from k_gen_first: only a block with some waits for it
  if (cl1 > cl0) dep_wait();
#pragma unroll 2
  for (int j = cl0; j < cl1; ++j) {
    const int c = __ldg(&P.gcl[j]);
    const double sgn = (c & 1) ? -1.0 : 1.0;
    const double* B = P.kcoh + (c >> 1);
#pragma unroll
    for (int i = 0; i < D2; ++i) acc[i] += sgn * B[i];
  }
  // the block's values: row q of the node, columns of the slot's DOFs (free ones in the row's F
  // block, constrained ones in its C block)
#pragma unroll
  for (int q = 0; q < DIM; ++q) {
    const bool rf = rrow[q] < P.n_free;
    double* vF = P.val[rf ? 0 : 2] + rF[q] + pre;
    double* vC = P.val[rf ? 1 : 3] + rC[q] + (slot * DIM - pre);
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      if (mk & (1 << d)) *vF++ = acc[q * DIM + d];
      else *vC++ = acc[q * DIM + d];
    }
  }
}

// The cohesive traction of entry j of a general node's traction list (zero when j >= j1).
template <int DIM, int L>
__device__ __forceinline__ void gen_traction(const DevProblem& P, int j, int j1, double* tk) {
#pragma unroll
  for (int q = 0; q < DIM; ++q) tk[q] = 0.0;
  if (j < j1) {
    const int c = __ldg(&P.gnode_tl[j]);
    const double sgn = (c & 1) ? -1.0 : 1.0;
    const double* tp = P.kcoh + (c >> 1);
#pragma unroll
    for (int q = 0; q < DIM; ++q) tk[q] = sgn * tp[q];
  }
}
// Residual of general node `node` by a group of L lanes (lane g): each part's terms are formed in
// parallel and summed in a fixed order with shuffles -- the static part in slot order, its
// macroscale response, then the tractions in adjacency order -- so the result does not depend on
// L.  The static part reads set-up data and U only, so it is summed before the wait for the
// kernel that forms the cohesive blocks (a programmatic dependent launch: see k_gen_rows).
// `valid` is uniform over the group.
template <int DIM, int L>
__device__ __forceinline__ void gen_resid(const DevProblem& P, int node, bool valid) {
  constexpr int NV = (DIM == 2) ? 3 : 6;
  if (!valid) return;
  const int g = threadIdx.x % L;
  const unsigned gmask = (L >= 32) ? 0xffffffffu : (((1u << L) - 1u) << ((threadIdx.x & 31) / L * L));
  const int t0 = __ldg(&P.gnode_tl_off[node]), t1 = __ldg(&P.gnode_tl_off[node + 1]);
  const int gdof = (g < DIM) ? __ldg(&P.growd[(size_t)node * 3 * DIM + g]) : 0;
  double tk[DIM];
  double r[DIM];
  const int4 gd = __ldg(&P.gdesc[node]);
  static_resid_group<DIM, L>(P, node, gd.w, g, gmask, r);
  if (P.subscale) {
    const double* Gs = P.stat_g + (size_t)node * DIM * NV;
#pragma unroll
    for (int q = 0; q < DIM; ++q)
#pragma unroll
      for (int v = 0; v < NV; ++v) r[q] += __ldg(&Gs[q * NV + v]) * P.eps_macro[v];
  }
  if (t1 > t0) dep_wait();   // the tractions come from k_gen_first
  for (int j0 = t0; j0 < t1; j0 += L) {
    gen_traction<DIM, L>(P, j0 + g, t1, tk);
    const int n_here = min(L, t1 - j0);
    for (int jj = 0; jj < n_here; ++jj)
#pragma unroll
      for (int q = 0; q < DIM; ++q) r[q] += __shfl_sync(gmask, tk[q], jj, L);
  }
  if (g >= DIM) return;
  double mine = r[0];
#pragma unroll
  for (int q = 1; q < DIM; ++q) if (g == q) mine = r[q];
  if (gdof < P.n_free) P.Pf[gdof] = mine; else P.Pp[gdof - P.n_free] = mine;
}

constexpr int kGenResidLanes = 8;   // lanes per node of the residual pass

// The cohesive elements (k_coh_elements' lanes); the general rows launched after it may start
// while it runs (programmatic dependent launch).
template <int DIM>
__global__ void __launch_bounds__(128) k_gen_first(DevProblem P) {
  dep_launch();
  constexpr int CQ = CohLanes<DIM>::CQ;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int ce = t / CQ;
  coh_element<DIM>(P, ce, t % CQ, ce < P.n_coh_el);
}

// The residuals and the blocks of the general rows in one launch: blocks [0, res_blocks) take
// the lane groups of nodes [n0, n1) (the longer chains of loads, so they are dispatched first),
// the rest the (node, slot) blocks [b0, b1).
template <int DIM>
__global__ void __launch_bounds__(128) k_gen_rows(DevProblem P, int n0, int n1, int res_blocks, int b0, int b1) {
  if ((int)blockIdx.x < res_blocks) {
    const int node = n0 + (blockIdx.x * blockDim.x + threadIdx.x) / kGenResidLanes;
    gen_resid<DIM, kGenResidLanes>(P, node, node < n1);
  } else {
    const int b = b0 + (blockIdx.x - res_blocks) * blockDim.x + threadIdx.x;
    if (b < b1) gen_block<DIM>(P, b);
  }
}

// ---------------------------------------------------------------- multi-strain residuals
// The residuals of the P.n_cases macroscale strains of general node `node` by a group of L lanes:
// for each case the operations of gen_resid with that case as the macroscale strain, in the same
// order -- the static part (formed once) and the case's macroscale response, then the tractions
// (the same for every case) -- so each case's values are those of the single-strain assembly.
template <int DIM, int L>
__device__ __forceinline__ void gen_resid_cases(const DevProblem& P, int node, bool valid) {
  constexpr int NV = (DIM == 2) ? 3 : 6;
  constexpr int MC = 6;
  if (!valid) return;
  const int nc = P.n_cases;
  const int g = threadIdx.x % L;
  const unsigned gmask = (L >= 32) ? 0xffffffffu : (((1u << L) - 1u) << ((threadIdx.x & 31) / L * L));
  const int t0 = __ldg(&P.gnode_tl_off[node]), t1 = __ldg(&P.gnode_tl_off[node + 1]);
  const int gdof = (g < DIM) ? __ldg(&P.growd[(size_t)node * 3 * DIM + g]) : 0;
  double rs[MC][DIM];
  {
    const int4 gd = __ldg(&P.gdesc[node]);
    double su[DIM];
    static_resid_group<DIM, L>(P, node, gd.w, g, gmask, su);
    const double* Gs = P.stat_g + (size_t)node * DIM * NV;
#pragma unroll
    for (int c = 0; c < MC; ++c) {
      if (c >= nc) break;
#pragma unroll
      for (int q = 0; q < DIM; ++q) {
        double v = su[q];
#pragma unroll
        for (int w = 0; w < NV; ++w) v += __ldg(&Gs[q * NV + w]) * P.eps_cases[c][w];
        rs[c][q] = v;
      }
    }
  }
  for (int j0 = t0; j0 < t1; j0 += L) {
    double tk[DIM];
    gen_traction<DIM, L>(P, j0 + g, t1, tk);
    const int n_here = min(L, t1 - j0);
    for (int jj = 0; jj < n_here; ++jj)
#pragma unroll
      for (int q = 0; q < DIM; ++q) {
        const double t = __shfl_sync(gmask, tk[q], jj, L);
#pragma unroll
        for (int c = 0; c < MC; ++c) if (c < nc) rs[c][q] += t;
      }
  }
  if (g >= DIM) return;
#pragma unroll
  for (int c = 0; c < MC; ++c) {
    if (c >= nc) break;
    double mine = rs[c][0];
#pragma unroll
    for (int q = 1; q < DIM; ++q) if (g == q) mine = rs[c][q];
    if (gdof < P.n_free) P.Pf_cases[(size_t)c * P.n_free + gdof] = mine;
    else P.Pp_cases[(size_t)c * P.n_const + gdof - P.n_free] = mine;
  }
}

template <int DIM>
__global__ void __launch_bounds__(128) k_gen_resid_cases(DevProblem P) {
  const int node = (blockIdx.x * blockDim.x + threadIdx.x) / kGenResidLanes;
  gen_resid_cases<DIM, kGenResidLanes>(P, node, node < P.n_slow_dn);
}

}  // namespace pgd
