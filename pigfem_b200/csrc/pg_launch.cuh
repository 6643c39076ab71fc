// pg_launch.cuh -- the launches of one assembly, one set-up pass and one multi-strain residual
// pass for a given dimension.  Instantiated once per dimension (pg_launch2.cu, pg_launch3.cu) so
// the two sets of kernels compile in separate translation units; pg_capi.cu calls them through
// the declarations below.
#pragma once

#include "pg_ctx.h"

namespace pgl {

// The kernels of one assembly (cohesive elements, stencil rows, general rows) on the context's
// streams, with the timing events of pg_kernel_times; P is the launch's problem view.
template <int DIM>
void assembly(pg_ctx* c, const pgd::DevProblem& P, bool jac, bool fp32);
// Set-up: the cut elements' volumetric blocks and macroscale-strain responses, on the allocation
// stream.
template <int DIM>
void cut_volumetric(pg_ctx* c, const pgd::DevProblem& P, double* gmac);
// Set-up: the static part of the general rows (k_general_static) on the allocation stream, after
// cut_volumetric.
template <int DIM>
void general_static(pg_ctx* c, const pgd::DevProblem& P, double* stat, double* stat_g);
// The residuals of P.n_cases macroscale strains (pg_residual_strains) on the context's stream.
template <int DIM>
void residual_cases(pg_ctx* c, const pgd::DevProblem& P);

#ifdef PG_LAUNCH_IMPL
template <int DIM>
void assembly(pg_ctx* c, const pgd::DevProblem& P, bool jac, bool fp32) {
  // fork: the fast rows (uncut elements only) run on the side stream, concurrently with the
  // cut-element kernels and the general rows on the main stream
  cudaEventRecord(c->ev[0], c->stream);
  cudaStreamWaitEvent(c->side, c->ev[0], 0);
  if (P.n_coh_el > 0) {
    const int tpb = 128;
    const int lanes = pgd::CohLanes<DIM>::CQ;
    const int grid = (int)(((long long)P.n_coh_el * lanes + tpb - 1) / tpb);
    pgd::k_coh_elements<DIM><<<grid, tpb, 0, c->stream>>>(P);
  }
  // 2D: the stencil rows run on the side stream, concurrently with the cohesive elements and the
  // general rows (the cohesive kernel leaves most SMs idle).  3D: on the main stream between the
  // two -- the 3D stencil and general kernels each fill the GPU, and run concurrently they took
  // 1.65 ms per 64^3 assembly against 1.0 ms one after the other.
  cudaEventRecord(c->ev[3], c->stream);
  cudaStream_t sst = (DIM == 2) ? c->side : c->stream;
  if (c->n_stencil > 0 && !jac) {
    const int tpb = 128;
    const int grid = (c->n_stencil + tpb - 1) / tpb;
    pgd::k_rows_stencil<DIM, double, false><<<grid, tpb, 0, sst>>>(P, c->grid, c->stencil, c->n_stencil);
  } else if (c->n_stencil > 0) {
    const int tpb = 128;
    const int nthreads = (DIM == 2) ? c->n_stencil : 3 * 32 * ((c->n_stencil + 31) / 32);
    const int grid = (nthreads + tpb - 1) / tpb;
    const size_t smem = (DIM == 2) ? pgd::stencil_stage_bytes(tpb) : 0;
    if (fp32) pgd::k_rows_stencil<DIM, float><<<grid, tpb, smem, sst>>>(P, c->grid, c->stencil, c->n_stencil);
    else pgd::k_rows_stencil<DIM, double><<<grid, tpb, smem, sst>>>(P, c->grid, c->stencil, c->n_stencil);
  }
  cudaEventRecord(c->ev[1], sst);
  if (P.n_slow_dn > 0 && !jac) {
    // residual only: entry-parallel groups of L lanes per node
    constexpr int L = 8;
    const int grid = (int)(((long long)P.n_slow_dn * L + 127) / 128);
    pgd::k_rows_general_resid<DIM, L><<<grid, 128, 0, c->stream>>>(P);
  } else if (P.n_slow_dn > 0) {
    const int slots = P.maxnb_general;
    constexpr int G = (DIM == 2) ? 4 : 8;
    const int grid = (P.n_slow_dn + (128 / G) - 1) / (128 / G);
    const size_t smem = (size_t)(128 / G) * pgd::general_slab_doubles(slots, DIM, P.max_mn) * sizeof(double);
    cudaFuncSetAttribute(pgd::k_rows_general<DIM, G>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    pgd::k_rows_general<DIM, G><<<grid, 128, smem, c->stream>>>(P, slots, P.max_mn);
  }
  cudaEventRecord(c->ev[4], c->stream);
  // join
  cudaStreamWaitEvent(c->stream, c->ev[1], 0);
  cudaEventRecord(c->ev[5], c->stream);
}

template <int DIM>
void cut_volumetric(pg_ctx* c, const pgd::DevProblem& P, double* gmac) {
  for (int cls = 0; cls < 2; ++cls) {
    const int n = c->n_cut_list[cls];
    if (n == 0) continue;
    const size_t smem = (size_t)pgd::cut_smem_doubles(c->cut_cls_qp[cls], c->cut_cls_nodes[cls], DIM) * sizeof(double);
    cudaFuncSetAttribute(pgd::k_cut_volumetric<DIM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    pgd::k_cut_volumetric<DIM><<<n, 64, smem, c->up>>>(P, c->cut_list[cls], n, gmac);
  }
}

template <int DIM>
void general_static(pg_ctx* c, const pgd::DevProblem& P, double* stat, double* stat_g) {
  if (P.n_stat > 0) pgd::k_general_static<DIM><<<(P.n_stat + 127) / 128, 128, 0, c->up>>>(P, stat, stat_g);
}

template <int DIM>
void residual_cases(pg_ctx* c, const pgd::DevProblem& P) {
  // the cohesive elements once (openings, laws, internal variables, tractions: U only), then
  // the stencil rows and the general rows for every case
  if (P.n_coh_el > 0) {
    const int lanes = pgd::CohLanes<DIM>::CQ;
    const int grid = (int)(((long long)P.n_coh_el * lanes + 127) / 128);
    pgd::k_coh_elements<DIM><<<grid, 128, 0, c->stream>>>(P);
  }
  if (c->n_stencil > 0) {
    const int grid = (c->n_stencil + 127) / 128;
    pgd::k_rows_stencil_cases<DIM><<<grid, 128, 0, c->stream>>>(P, c->grid, c->stencil, c->n_stencil);
  }
  if (P.n_slow_dn > 0) {
    constexpr int L = 8;
    const int grid = (int)(((long long)P.n_slow_dn * L + 127) / 128);
    pgd::k_rows_general_cases<DIM, L><<<grid, 128, 0, c->stream>>>(P);
  }
}

#define PG_INSTANTIATE_LAUNCHES(D)                                                     \
  template void assembly<D>(pg_ctx*, const pgd::DevProblem&, bool, bool);              \
  template void cut_volumetric<D>(pg_ctx*, const pgd::DevProblem&, double*);           \
  template void general_static<D>(pg_ctx*, const pgd::DevProblem&, double*, double*);  \
  template void residual_cases<D>(pg_ctx*, const pgd::DevProblem&);
#endif

}  // namespace pgl
