// pg_launch.cuh -- the launches of one assembly, one set-up pass and one multi-strain residual
// pass for a given dimension.  Instantiated once per dimension (pg_launch2.cu, pg_launch3.cu) so
// the two sets of kernels compile in separate translation units; pg_capi.cu calls them through
// the declarations below.
#pragma once

#include "pg_ctx.h"
#include "pg_tile.cuh"
#include "pg_general.cuh"

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
// Set-up: the 2D tiles' shape constants (k_tile2_consts) into P, on the allocation stream; a no-op
// in 3D or without tiles.  0, or 1 when a CUDA call fails.
template <int DIM>
int tile_consts(pg_ctx* c, pgd::DevProblem& P);

#ifdef PG_LAUNCH_IMPL
template <int DIM>
void assembly(pg_ctx* c, const pgd::DevProblem& P, bool jac, bool fp32) {
  const bool func = (P.flags & PG_FUNC) != 0;
  auto blocks_of = [](long long n) { return (int)((n + 127) / 128); };
  const bool simplex_general = P.n_slow_dn > 0 && P.npe == DIM + 1;
  // 2D: the general chain (cohesive elements, element records, general rows) runs on the
  // high-priority stream side2 and the structured tiles on the low-priority stream side, both
  // from the fork: the block scheduler dispatches the chain's blocks first, and the tiles fill
  // the rest of the GPU.  3D: all on the main stream, cohesive elements and records, the tiles,
  // then the general rows (the 3D tile and general kernels each fill the GPU).
  cudaEventRecord(c->ev[0], c->stream);
  cudaStreamWaitEvent(c->side, c->ev[0], 0);
  cudaStreamWaitEvent(c->side2, c->ev[0], 0);
  cudaStream_t gst = (DIM == 2) ? c->side2 : c->stream;
  cudaStream_t sst = (DIM == 2) ? c->side : c->stream;
  {
    const int coh_blocks = (P.n_coh_el > 0) ? blocks_of((long long)P.n_coh_el * pgd::CohLanes<DIM>::CQ) : 0;
    if (coh_blocks > 0) pgd::k_gen_first<DIM><<<coh_blocks, 128, 0, gst>>>(P);
  }
  // (the timing event between the cohesive/record kernel and the general rows is recorded only
  // when timing: an event between them would hold back the general rows' early start)
  if (c->timing) cudaEventRecord(c->ev[3], gst);
  c->timed_last = c->timing;
  if (DIM == 2 && c->n_tiles > 0) {
    // 2D: one CTA per 16 x 8 tile of grid nodes, each element formed once (pg_tile.cuh)
    const size_t smem = pgd::tile2_smem_bytes();
    if (!jac) pgd::k_rows_tile2<double, false><<<c->n_tiles, pgd::kTileThreads, smem, sst>>>(P, c->grid, c->tiles, c->tnodes, c->tsegs);
    else if (fp32) pgd::k_rows_tile2<float, true><<<c->n_tiles, pgd::kTileThreads, smem, sst>>>(P, c->grid, c->tiles, c->tnodes, c->tsegs);
    else pgd::k_rows_tile2<double, true><<<c->n_tiles, pgd::kTileThreads, smem, sst>>>(P, c->grid, c->tiles, c->tnodes, c->tsegs);
  } else if (DIM == 3 && c->n_tiles > 0) {
    // 3D: one CTA per 4 x 4 x 4 tile of grid nodes, each tet formed once (pg_tile.cuh)
    const size_t smem = pgd::tile3_smem_bytes();
    if (!jac) {
      cudaFuncSetAttribute(pgd::k_rows_tile3<double, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      pgd::k_rows_tile3<double, false><<<c->n_tiles, pgd::kT3Threads, smem, sst>>>(P, c->grid, c->tiles, c->tnodes, c->tsegs, *c->t3c);
    } else if (fp32) {
      cudaFuncSetAttribute(pgd::k_rows_tile3<float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      pgd::k_rows_tile3<float, true><<<c->n_tiles, pgd::kT3Threads, smem, sst>>>(P, c->grid, c->tiles, c->tnodes, c->tsegs, *c->t3c);
    } else {
      cudaFuncSetAttribute(pgd::k_rows_tile3<double, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      pgd::k_rows_tile3<double, true><<<c->n_tiles, pgd::kT3Threads, smem, sst>>>(P, c->grid, c->tiles, c->tnodes, c->tsegs, *c->t3c);
    }
  } else if (c->n_stencil > 0 && !jac) {
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
  if (simplex_general) {
    // block-parallel general rows (pg_general.cuh): residual lane groups and blocks in one launch
    const int res_blocks = func ? blocks_of((long long)P.n_slow_dn * pgd::kGenResidLanes) : 0;
    const int blk_blocks = jac ? blocks_of(P.n_gblk) : 0;
    if (res_blocks + blk_blocks > 0) {
      // programmatic dependent launch: the general rows' blocks start while the kernel before them
      // in the stream finishes, load their descriptors and static parts, and wait in the kernel
      // (griddepcontrol.wait) before reading that kernel's output
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3((unsigned)(res_blocks + blk_blocks));
      cfg.blockDim = dim3(128);
      cfg.dynamicSmemBytes = 0;
      cfg.stream = gst;
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
      at[0].val.programmaticStreamSerializationAllowed = 1;
      cfg.attrs = at;
      cfg.numAttrs = 1;
      cudaLaunchKernelEx(&cfg, pgd::k_gen_rows<DIM>, P, 0, P.n_slow_dn, res_blocks, 0, P.n_gblk);
    }
  } else if (P.n_slow_dn > 0 && !jac) {
    // quad4 meshes, residual only: entry-parallel groups of L lanes per node
    constexpr int L = 8;
    const int grid = (int)(((long long)P.n_slow_dn * L + 127) / 128);
    pgd::k_rows_general_resid<DIM, L, (DIM == 2) ? 4 : DIM + 1><<<grid, 128, 0, gst>>>(P);
  } else if (P.n_slow_dn > 0 && DIM == 2) {
    // quad4 meshes: a lane group per general node (every node is one)
    const int slots = P.maxnb_general;
    constexpr int L = 8;
    const int grid = (P.n_slow_dn + (128 / L) - 1) / (128 / L);
    const size_t smem = (size_t)(128 / L) * pgd::general_slab_doubles(slots, DIM, L, 4) * sizeof(double);
    cudaFuncSetAttribute(pgd::k_rows_general<DIM, L, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    pgd::k_rows_general<DIM, L, 4><<<grid, 128, smem, gst>>>(P, slots, 0, P.n_slow_dn);
  }
  cudaEventRecord(c->ev[4], gst);
  // join
  cudaStreamWaitEvent(c->stream, c->ev[1], 0);
  cudaStreamWaitEvent(c->stream, c->ev[4], 0);
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
    // a lane group per general node sums each case's residual as the single-strain assembly does
    const int grid = (int)(((long long)P.n_slow_dn * pgd::kGenResidLanes + 127) / 128);
    pgd::k_gen_resid_cases<DIM><<<grid, 128, 0, c->stream>>>(P);
  }
}

template <int DIM>
int tile_consts(pg_ctx* c, pgd::DevProblem& P) {
  if (c->n_tiles == 0) return 0;
  const pg::ProblemDesc& d = c->s.desc;
  if (DIM == 3) {
    // the 3D shapes into a host copy (the single launches' kernel parameter) and a device copy
    // (read by the batched launches)
    const double hx = (d.hi[0] - d.lo[0]) / d.n[0], hy = (d.hi[1] - d.lo[1]) / d.n[1], hz = (d.hi[2] - d.lo[2]) / d.n[2];
    pgd::Tile3Const* dc = nullptr;
    if (cudaMallocAsync(&dc, sizeof(pgd::Tile3Const), c->up) != cudaSuccess) return 1;
    pg_track_alloc(c, dc, sizeof(pgd::Tile3Const));
    pgd::k_tile3_consts<DIM><<<1, 32, 0, c->up>>>(P, d.lo[0], d.lo[1], d.lo[2], hx, hy, hz, dc);
    if (!c->t3c) c->t3c = new pgd::Tile3Const;
    cudaMemcpyAsync(c->t3c, dc, sizeof(pgd::Tile3Const), cudaMemcpyDeviceToHost, c->up);
    if (cudaStreamSynchronize(c->up) != cudaSuccess) return 1;
    c->d_t3c = dc;
    return 0;
  }
  const double hx = (d.hi[0] - d.lo[0]) / d.n[0], hy = (d.hi[1] - d.lo[1]) / d.n[1];
  constexpr int n_out = 24 + 4 + 2 * 432;
  double* dout = nullptr;
  if (cudaMallocAsync(&dout, n_out * sizeof(double), c->up) != cudaSuccess) return 1;
  pgd::k_tile2_consts<DIM><<<1, 32, 0, c->up>>>(P, d.lo[0], d.lo[1], hx, hy, dout);
  std::vector<double> h(n_out);
  cudaMemcpyAsync(h.data(), dout, n_out * sizeof(double), cudaMemcpyDeviceToHost, c->up);
  cudaFreeAsync(dout, c->up);
  if (cudaStreamSynchronize(c->up) != cudaSuccess) return 1;
  for (int sh = 0; sh < 4; ++sh) {
    for (int n = 0; n < 3; ++n) { P.tile_g[sh][n][0] = h[sh * 6 + n * 2]; P.tile_g[sh][n][1] = h[sh * 6 + n * 2 + 1]; }
    P.tile_w[sh] = h[24 + sh];
    for (int m = 0; m < 3; ++m)
      for (int i = 0; i < 36; ++i) {
        P.tile_ke[sh][m][i] = h[28 + (sh * 3 + m) * 36 + i];
        P.tile_kef[sh][m][i] = (float)h[28 + 432 + (sh * 3 + m) * 36 + i];
      }
  }
  return 0;
}

#define PG_INSTANTIATE_LAUNCHES(D)                                                     \
  template void assembly<D>(pg_ctx*, const pgd::DevProblem&, bool, bool);              \
  template void cut_volumetric<D>(pg_ctx*, const pgd::DevProblem&, double*);           \
  template void general_static<D>(pg_ctx*, const pgd::DevProblem&, double*, double*);  \
  template void residual_cases<D>(pg_ctx*, const pgd::DevProblem&);                    \
  template int tile_consts<D>(pg_ctx*, pgd::DevProblem&);
#endif

}  // namespace pgl
