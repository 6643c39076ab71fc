// pg_general.cuh -- block-parallel general rows (tri3 / tet4 meshes).
//
// The general rows are the DOF nodes the structured tiles do not take: boundary rows, nodes of
// cut elements and enrichment nodes.  Their values are formed in three passes whose loads are
// all independent of one another (the set-up flattened every index), so each thread's chain of
// memory round trips is short:
//   gen_records  one thread per uncut element adjacent to a general node: geometry (gradients,
//                J W) from the node coordinates and the stress from U (+ eps_macro), once, into
//                the element's record (GenRec);
//   gen_block    one thread per (general node, neighbour slot) block: the static part (the cut
//                elements' volumetric blocks reduced at set-up), the cohesive blocks of the
//                cohesive elements holding both nodes (kcoh, from k_coh_elements) and the uncut
//                elements holding both (w B_la^T D B_lb from the records), in adjacency order;
//                then the block's CSR values, each written once;
//   gen_resid    a group of 8 lanes per general node: the static part times the displacements
//                (slot order) and the macroscale-strain response, the cohesive tractions and the
//                uncut elements' w B_la^T sigma (adjacency order), terms formed in parallel and
//                summed in that order by shuffles.
// Every value is a sum in a fixed order, so results are bit-reproducible.  Residual-only
// assemblies run gen_records and gen_resid alone, so their residuals are bitwise those of the full
// assembly.  An assembly launches the passes as two kernels: k_gen_first (the cohesive elements
// and the records) and k_gen_rows (residuals and blocks).
#pragma once

#include "pg_stencil.cuh"

namespace pgd {

// Element record: gradients g[k][d] at k * DIM + d, the weight J W, the stress, the material
// (as a double), padded to whole 32-byte sectors -- 12 doubles (96 B) for tri3, 20 (160 B) for
// tet4 -- so the rows' scattered reads of a record touch two or three sectors.
template <int DIM>
struct GenRec {
  static constexpr int NPE = DIM + 1, NV = (DIM == 2) ? 3 : 6;
  static constexpr int W = NPE * DIM, SIG = W + 1, MAT = SIG + NV;
  static constexpr int STRIDE = (DIM == 2) ? 12 : 20;
};
template <int DIM>
__host__ __device__ constexpr int gen_fields() { return GenRec<DIM>::STRIDE; }

// Programmatic dependent launch: k_gen_rows may start while the kernel before it in the stream
// (k_gen_first in 2D, the tiles in 3D) still runs; griddepcontrol.wait returns once that grid has
// completed and its writes are visible (at once when the launch had no such dependency), so
// everything read after it -- the cohesive blocks and the element records -- is complete.
__device__ __forceinline__ void dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
// Lets the dependent grid launch now (its blocks then do their independent loads).
__device__ __forceinline__ void dep_launch() { asm volatile("griddepcontrol.launch_dependents;" :::); }

// The record of element record r into o[0 .. STRIDE).  STRAIN: the stress slots hold the strain
// of U alone (no macroscale part), for the multi-strain pass.
template <int DIM, bool STRAIN = false>
__device__ __forceinline__ void gen_record_values(const DevProblem& P, int r, double* o) {
  constexpr int NPE = DIM + 1;
  constexpr int NV = (DIM == 2) ? 3 : 6;
  using R = GenRec<DIM>;
  const int4 nodes = __ldg(&P.grec_nodes[r]);
  const int nd[4] = {nodes.x, nodes.y, nodes.z, nodes.w};
  double x[NPE][DIM], u[NPE][DIM], g[NPE][DIM], J;
#pragma unroll
  for (int k = 0; k < NPE; ++k) { load_node<DIM>(P.X, nd[k], x[k]); load_node<DIM>(P.U, nd[k], u[k]); }
  simplex_geom<DIM, double>(x, g, &J);
  const double wgt = J * ((DIM == 2) ? tri4_wsum() : tet5_wsum());
  double eps[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) eps[v] = 0.0;
#pragma unroll
  for (int k = 0; k < NPE; ++k) add_strain<DIM, double>(g[k], u[k], eps);
  if (!STRAIN && P.subscale) {
#pragma unroll
    for (int v = 0; v < NV; ++v) eps[v] += P.eps_macro[v];
  }
  // sigma = D eps over D's nonzero pattern (every bulk material has the isotropic one), D read
  // from device memory: a per-thread material index into the parameter block would be serialized
  double sig[NV], dm[(DIM == 2) ? 5 : 12];
  const int m = __ldg(&P.grec_mat[r]);
  if (STRAIN) {
#pragma unroll
    for (int v = 0; v < NV; ++v) sig[v] = eps[v];
  } else {
    iso_d<DIM, double>(P, m, dm);
    lei_stress_iso<DIM, double>(dm, eps, sig);
  }
#pragma unroll
  for (int k = 0; k < NPE; ++k)
#pragma unroll
    for (int d = 0; d < DIM; ++d) o[k * DIM + d] = g[k][d];
  o[R::W] = wgt;
#pragma unroll
  for (int v = 0; v < NV; ++v) o[R::SIG + v] = sig[v];
  o[R::MAT] = (double)m;
#pragma unroll
  for (int f = R::MAT + 1; f < R::STRIDE; ++f) o[f] = 0.0;
}

template <int DIM>
__device__ __forceinline__ void gen_record(const DevProblem& P, int r) {
  constexpr int S = GenRec<DIM>::STRIDE;
  double o[S];
  gen_record_values<DIM>(P, r, o);
  double* dst = P.grec + (size_t)r * S;
#pragma unroll
  for (int f = 0; f < S; ++f) dst[f] = o[f];
}

template <int DIM>
__device__ __forceinline__ void gen_block(const DevProblem& P, int b) {
  constexpr int D2 = DIM * DIM;
  constexpr int NV = (DIM == 2) ? 3 : 6;
  using R = GenRec<DIM>;
  const int4 bd = __ldg(&P.gblk[b]);
  const int ul1 = __ldg(&P.gblk[b + 1].w);
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
  if (bd.z >= 0) {
    const double* S = P.stat + (size_t)bd.z * D2;
#pragma unroll
    for (int i = 0; i < D2; ++i) acc[i] = __ldg(&S[i]);
  } else {
#pragma unroll
    for (int i = 0; i < D2; ++i) acc[i] = 0.0;
  }
  dep_wait();   // the cohesive blocks and element records below come from k_gen_first
#pragma unroll 2
  for (int j = cl0; j < cl1; ++j) {
    const int c = __ldg(&P.gcl[j]);
    const double sgn = (c & 1) ? -1.0 : 1.0;
    const double* B = P.kcoh + (c >> 1);
#pragma unroll
    for (int i = 0; i < D2; ++i) acc[i] += sgn * B[i];
  }
#pragma unroll 4
  for (int j = bd.w; j < ul1; ++j) {
    const int c = __ldg(&P.gul[j]);
    const int r = c >> 4, la = (c >> 2) & 3, lb = c & 3;
    const double* o = P.grec + (size_t)r * R::STRIDE;
    double ga[DIM], gb[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) { ga[d] = o[la * DIM + d]; gb[d] = o[lb * DIM + d]; }
    const double w = o[R::W];
    // D's nonzero pattern from device memory (see gen_record); part_iso forms the same values as
    // bt_d_row over the full D (the terms it leaves out are exact zeros)
    double dm[(DIM == 2) ? 5 : 12];
    iso_d<DIM, double>(P, (int)o[R::MAT], dm);
#pragma unroll
    for (int q = 0; q < DIM; ++q) {
      double part[NV];
      part_iso<DIM, double>(dm, ga, q, part);
#pragma unroll
      for (int q2 = 0; q2 < DIM; ++q2) acc[q * DIM + q2] += w * part_b<DIM, double>(part, gb, q2);
    }
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

// Residual of general node `node` by a group of L lanes (lane g): each part's terms are formed in
// parallel and summed in a fixed order with shuffles -- the static part in slot order, then the
// tractions and the uncut elements in adjacency order -- so the result does not depend on L.
// `valid` is uniform over the group.
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
template <int DIM, int L>
__device__ __forceinline__ void gen_uncut_force(const DevProblem& P, int j, int j1, double* rv) {
  constexpr int NV = (DIM == 2) ? 3 : 6;
  using R = GenRec<DIM>;
#pragma unroll
  for (int q = 0; q < DIM; ++q) rv[q] = 0.0;
  if (j < j1) {
    const int c = __ldg(&P.gnode_ul[j]);
    const int rec = c >> 2, la = c & 3;
    const double* o = P.grec + (size_t)rec * R::STRIDE;
    double ga[DIM], sig[NV];
#pragma unroll
    for (int d = 0; d < DIM; ++d) ga[d] = o[la * DIM + d];
    const double w = o[R::W];
#pragma unroll
    for (int v = 0; v < NV; ++v) sig[v] = o[R::SIG + v];
#pragma unroll
    for (int q = 0; q < DIM; ++q) rv[q] = w * bt_sig<DIM, double>(ga, sig, q);
  }
}

// Residual of general node `node` by a group of L lanes (lane g): each part's terms are formed in
// parallel and summed in a fixed order with shuffles -- the static part in slot order, then the
// tractions and the uncut elements in adjacency order -- so the result does not depend on L.  The
// static part reads set-up data and U only, so it is summed before the wait for the kernel that
// forms the cohesive blocks and element records (a programmatic dependent launch: see
// k_gen_rows).  `valid` is uniform over the group.
template <int DIM, int L>
__device__ __forceinline__ void gen_resid(const DevProblem& P, int node, bool valid) {
  constexpr int NV = (DIM == 2) ? 3 : 6;
  if (!valid) { dep_wait(); return; }
  const int g = threadIdx.x % L;
  const unsigned gmask = (L >= 32) ? 0xffffffffu : (((1u << L) - 1u) << ((threadIdx.x & 31) / L * L));
  const int t0 = __ldg(&P.gnode_tl_off[node]), t1 = __ldg(&P.gnode_tl_off[node + 1]);
  const int u0 = __ldg(&P.gnode_ul_off[node]), u1 = __ldg(&P.gnode_ul_off[node + 1]);
  const int gdof = (g < DIM) ? __ldg(&P.growd[(size_t)node * 3 * DIM + g]) : 0;
  double tk[DIM], rv[DIM];
  double r[DIM];
#pragma unroll
  for (int q = 0; q < DIM; ++q) r[q] = 0.0;
  if (node < P.n_stat) {
    const int4 gd = __ldg(&P.gdesc[node]);
    static_resid_group<DIM, L>(P, node, gd.w, g, gmask, r);
    if (P.subscale) {
      const double* Gs = P.stat_g + (size_t)node * DIM * NV;
#pragma unroll
      for (int q = 0; q < DIM; ++q)
#pragma unroll
        for (int v = 0; v < NV; ++v) r[q] += __ldg(&Gs[q * NV + v]) * P.eps_macro[v];
    }
  }
  dep_wait();
  for (int j0 = t0; j0 < t1; j0 += L) {
    gen_traction<DIM, L>(P, j0 + g, t1, tk);
    const int n_here = min(L, t1 - j0);
    for (int jj = 0; jj < n_here; ++jj)
#pragma unroll
      for (int q = 0; q < DIM; ++q) r[q] += __shfl_sync(gmask, tk[q], jj, L);
  }
  for (int j0 = u0; j0 < u1; j0 += L) {
    gen_uncut_force<DIM, L>(P, j0 + g, u1, rv);
    const int n_here = min(L, u1 - j0);
    for (int jj = 0; jj < n_here; ++jj)
#pragma unroll
      for (int q = 0; q < DIM; ++q) r[q] += __shfl_sync(gmask, rv[q], jj, L);
  }
  if (g >= DIM) return;
  double mine = r[0];
#pragma unroll
  for (int q = 1; q < DIM; ++q) if (g == q) mine = r[q];
  if (gdof < P.n_free) P.Pf[gdof] = mine; else P.Pp[gdof - P.n_free] = mine;
}

constexpr int kGenResidLanes = 8;   // lanes per node of the residual pass

template <int DIM>
__global__ void __launch_bounds__(128) k_gen_records(DevProblem P) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < P.n_grec) gen_record<DIM>(P, r);
}
template <int DIM>
__global__ void __launch_bounds__(128) k_gen_blocks(DevProblem P, int b0, int b1) {
  const int b = b0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (b < b1) gen_block<DIM>(P, b);
}
template <int DIM>
__global__ void __launch_bounds__(128) k_gen_resid(DevProblem P, int n0, int n1) {
  const int node = n0 + (blockIdx.x * blockDim.x + threadIdx.x) / kGenResidLanes;
  gen_resid<DIM, kGenResidLanes>(P, node, node < n1);
}

// Records r0 .. r0 + 127 by a block of 128 threads: the block's records are contiguous, so they are
// staged in shared memory (an odd row pitch, so the per-thread rows meet no bank twice) and
// stored by the whole block, consecutive threads on consecutive addresses.
template <int DIM, bool STRAIN>
__device__ __forceinline__ void record_block(const DevProblem& P, int r0) {
  constexpr int S = GenRec<DIM>::STRIDE, SP = S + 1;
  __shared__ double st[128 * SP];
  const int r = r0 + threadIdx.x;
  if (r < P.n_grec) {
    double o[S];
    gen_record_values<DIM, STRAIN>(P, r, o);
#pragma unroll
    for (int f = 0; f < S; ++f) st[threadIdx.x * SP + f] = o[f];
  }
  __syncthreads();
  const int n = min((int)blockDim.x, P.n_grec - r0) * S;
  double* dst = P.grec + (size_t)r0 * S;
  for (int k = threadIdx.x; k < n; k += blockDim.x) dst[k] = st[(k / S) * SP + k % S];
}

// The cohesive elements and the element records in one launch (both read U and the geometry
// only): blocks [0, coh_blocks) take the cohesive quadrature lanes (k_coh_elements), the rest
// the records.
template <int DIM>
__global__ void __launch_bounds__(128) k_gen_first(DevProblem P, int coh_blocks) {
  dep_launch();
  if ((int)blockIdx.x < coh_blocks) {
    constexpr int CQ = CohLanes<DIM>::CQ;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int ce = t / CQ;
    coh_element<DIM>(P, ce, t % CQ, ce < P.n_coh_el);
  } else {
    record_block<DIM, false>(P, (blockIdx.x - coh_blocks) * blockDim.x);
  }
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
    else dep_wait();
  }
}

// ---------------------------------------------------------------- multi-strain residuals
// Records for pg_residual_strains: the stress slots hold the strain of U alone.
template <int DIM>
__global__ void __launch_bounds__(128) k_gen_records_strain(DevProblem P) {
  record_block<DIM, true>(P, blockIdx.x * blockDim.x);
}

// The residuals of the P.n_cases macroscale strains of general node `node` by a group of L lanes:
// for each case the operations of gen_resid with that case as the macroscale strain, in the same
// order -- the static part and its macroscale response, the tractions (the same for every case),
// then the uncut elements, whose stress is formed from the record's strain of U plus the case's
// strain -- so each case's values are those of the single-strain assembly.
template <int DIM, int L>
__device__ __forceinline__ void gen_resid_cases(const DevProblem& P, int node, bool valid) {
  constexpr int NV = (DIM == 2) ? 3 : 6;
  constexpr int MC = 6;
  using R = GenRec<DIM>;
  if (!valid) return;
  const int nc = P.n_cases;
  const int g = threadIdx.x % L;
  const unsigned gmask = (L >= 32) ? 0xffffffffu : (((1u << L) - 1u) << ((threadIdx.x & 31) / L * L));
  const int t0 = __ldg(&P.gnode_tl_off[node]), t1 = __ldg(&P.gnode_tl_off[node + 1]);
  const int u0 = __ldg(&P.gnode_ul_off[node]), u1 = __ldg(&P.gnode_ul_off[node + 1]);
  const int gdof = (g < DIM) ? __ldg(&P.growd[(size_t)node * 3 * DIM + g]) : 0;
  double rs[MC][DIM];
#pragma unroll
  for (int c = 0; c < MC; ++c)
#pragma unroll
    for (int q = 0; q < DIM; ++q) rs[c][q] = 0.0;
  if (node < P.n_stat) {
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
  for (int j0 = u0; j0 < u1; j0 += L) {
    double rv[MC][DIM];
#pragma unroll
    for (int c = 0; c < MC; ++c)
#pragma unroll
      for (int q = 0; q < DIM; ++q) rv[c][q] = 0.0;
    if (j0 + g < u1) {
      const int cc = __ldg(&P.gnode_ul[j0 + g]);
      const int rec = cc >> 2, la = cc & 3;
      const double* o = P.grec + (size_t)rec * R::STRIDE;
      double ga[DIM], eps[NV], dm[(DIM == 2) ? 5 : 12];
#pragma unroll
      for (int d = 0; d < DIM; ++d) ga[d] = o[la * DIM + d];
      const double w = o[R::W];
#pragma unroll
      for (int v = 0; v < NV; ++v) eps[v] = o[R::SIG + v];
      iso_d<DIM, double>(P, (int)o[R::MAT], dm);
#pragma unroll
      for (int c = 0; c < MC; ++c) {
        if (c >= nc) break;
        double ek[NV], sig[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) ek[v] = eps[v] + P.eps_cases[c][v];
        lei_stress_iso<DIM, double>(dm, ek, sig);
#pragma unroll
        for (int q = 0; q < DIM; ++q) rv[c][q] = w * bt_sig<DIM, double>(ga, sig, q);
      }
    }
    const int n_here = min(L, u1 - j0);
    for (int jj = 0; jj < n_here; ++jj)
#pragma unroll
      for (int c = 0; c < MC; ++c) {
        if (c >= nc) break;
#pragma unroll
        for (int q = 0; q < DIM; ++q) rs[c][q] += __shfl_sync(gmask, rv[c][q], jj, L);
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
