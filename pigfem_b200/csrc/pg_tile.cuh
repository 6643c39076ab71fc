// pg_tile.cuh -- tiled structured-grid rows: each element is formed once per tile.
//
// 2D (stencil_tile2).  The stencil nodes of a structured tri3 grid (pg_stencil.cuh) are grouped
// into tiles of 16 x 8 grid nodes.  One CTA of 256 threads takes a tile:
//   A. the coordinates and displacements of the tile's nodes and of a one-node halo (18 x 10)
//      go to shared memory;
//   B. every element of the 17 x 9 cells touching the tile (306 tri3) is formed once from them --
//      gradients, weight J W, stress -- into a shared record.  The element's nodes follow the
//      grid's union-jack split (the set-up checked every stencil node's elements against it);
//   C. one thread per stencil node and row q (lanes 2n and 2n + 1 of a warp hold rows 0 and 1 of
//      one node, so each record load serves both rows with one shared-memory access; warps 0-3 the
//      64 nodes of class 0 (8 elements), warps 4-7 the 64 of class 1 (4 elements)) sums its block
//      row and residual entry from the records in adjacency order -- the operations of
//      stencil_rows, with the geometry read instead of recomputed -- keeping the row in registers
//      and writing the residual entry;
//   D. the rows go to a shared stage laid out like the CSR (a tile row of grid nodes is one run
//      of the CSR when its nodes' rows are consecutive), and the CTA stores the set-up's
//      contiguous segments with consecutive threads on consecutive addresses.
// 3D (stencil_tile3): tiles of 4 x 4 x 4 grid nodes, one CTA of 192 threads (a thread per node
// and row, rows warp-uniform); the 750 tets of the 5 x 5 x 5 cells touching the tile (six per hex,
// the grid's split) are formed once into records; node 0's gradient is not stored but re-formed
// as the negated sum of the other three, as simplex_geom forms it.
// Node data and records are structure-of-arrays (2D: of double2 pairs, one 16-byte access each),
// with the element index permuted so that the lanes of a warp touch consecutive words both when
// the elements are formed and when the node rows read them (at most 2-way shared-memory bank
// conflicts).  Compared with one thread per node
// (and row) forming its own elements, every element's geometry, division and stress is computed
// once instead of three (2D) or twelve (3D) times, and the row stores need no shuffles.
#pragma once

#include "pg_stencil.cuh"

namespace pgd {

// ------------------------------------------------------------------ 2D
constexpr int kTileX = 16, kTileY = 8;                     // grid nodes per tile
constexpr int kTileNX = kTileX + 2, kTileNY = kTileY + 2;  // nodes with the halo
constexpr int kTileNodes2 = kTileNX * kTileNY;             // 180
constexpr int kTileCX = kTileX + 1, kTileCY = kTileY + 1;  // cells touching the tile
constexpr int kTileHX = (kTileCX + 1) / 2;                 // cell columns per parity (9)
// record slots per (element-in-cell, column parity) plane: the 81 cells of a plane padded to 84,
// so that within a quarter-warp of the element pass (8 consecutive cells, alternating planes)
// the two planes' 16-byte record stores fall in different banks
constexpr int kTilePlane = 84;
static_assert(kTilePlane >= kTileCY * kTileHX && kTilePlane % 8 == 4, "plane padding");
constexpr int kTileRecN = 2 * 2 * kTilePlane;              // record slots (336; 306 used)
constexpr int kTileFields = 12;                            // doubles per record slot (11 used)
constexpr int kTileRowStage = 8 * 36 + 8 * 20;             // doubles of a tile row's runs (448)
constexpr int kTileOwn = kTileX * kTileY;                  // the tile's own nodes (128)
constexpr int kTileThreads = 2 * kTileOwn;                 // a thread per node and row

// Record slot of element `sub` of tile cell (cx, cy): cells of one x parity are consecutive in x,
// so the class-uniform node warps (nodes two cells apart) read consecutive slots.
__host__ __device__ constexpr int tile2_slot(int cx, int cy, int sub) {
  return (sub * 2 + (cx & 1)) * kTilePlane + cy * kTileHX + (cx >> 1);
}

// Stage word a of a 2D tile is stored at a ^ ((a >> 4) & 3): a permutation inside each aligned
// group of 4 doubles, changing with the group of 16 the word falls in.  A half-warp's 8-byte row
// store writes one value of each of 8 nodes' two rows (runs 56 doubles apart, rows NN x 2 apart),
// which without it meet in 4 bank pairs (4 wavefronts per half-warp store); with it the stores
// average 1.6, and the warp-wide reads of a segment stay free of conflicts.
__host__ __device__ constexpr int tile2_swizzle(int a) { return a ^ ((a >> 4) & 3); }

__host__ __device__ constexpr size_t tile2_smem_bytes() {
  // node data (x, u as two double2 arrays) then the record fields; the stage reuses the record area
  return (size_t)(4 * kTileNodes2 + kTileFields * kTileRecN) * sizeof(double);
}
static_assert(kTileFields * kTileRecN >= kTileY * kTileRowStage, "the stage fits the record area");
static_assert((kTileY * kTileRowStage) % 4 == 0, "the swizzle stays inside the stage");

// Tile descriptor: {first node i, first node j, first segment, segment count}; per own node (class
// 0 nodes, then class 1) an entry {node id or -1, first free DOF, first CSR slot, stage offset};
// per segment {stage offset, first CSR slot, length, 0}.  Every thread of the CTA calls it.
template <typename T, bool JAC>
__device__ __forceinline__ void stencil_tile2(const DevProblem& P, const GridInfo& gi, int4 td,
                                              const int4* __restrict__ tnodes, const int4* __restrict__ segs,
                                              double* sm) {
  constexpr int NV = 3, ND = 5;
  constexpr int RN = kTileRecN;
  const int t = threadIdx.x;
  const int i0 = td.x, j0 = td.y;
  const int sx = gi.nx + 1;
  // shared memory as double2 pairs, so each pair is one 16-byte access: node coordinates and
  // displacements, then the record fields of slot k -- g0, g1, g2, (w, sigma_xx),
  // (sigma_yy, sigma_xy) at rec2[f * RN + k] -- and the material at recm[k]
  double2* xs = reinterpret_cast<double2*>(sm);
  double2* us = xs + kTileNodes2;
  double2* rec2 = us + kTileNodes2;
  double* recm = reinterpret_cast<double*>(rec2 + 5 * RN);
  double* rec = reinterpret_cast<double*>(rec2);       // the stage, after the records are consumed
  // A: nodes
  for (int k = t; k < kTileNodes2; k += kTileThreads) {
    const int i = i0 - 1 + k % kTileNX, j = j0 - 1 + k / kTileNX;
    if (i >= 0 && i <= gi.nx && j >= 0 && j <= gi.ny) {
      const int id = j * sx + i;
      xs[k] = __ldg(reinterpret_cast<const double2*>(P.X) + id);
      us[k] = __ldg(reinterpret_cast<const double2*>(P.U) + id);
    }
  }
  __syncthreads();
  // B: elements of the cells touching the tile, cell order (consecutive lanes read consecutive
  // nodes), each into its record slot
  for (int it = t; it < 2 * kTileCX * kTileCY; it += kTileThreads) {
    const int cx = it % kTileCX, cy = (it / kTileCX) % kTileCY, sub = it / (kTileCX * kTileCY);
    const int k = tile2_slot(cx, cy, sub);
    const int ci = i0 - 1 + cx, cj = j0 - 1 + cy;
    if (ci < 0 || ci >= gi.nx || cj < 0 || cj >= gi.ny) continue;
    // union-jack split of cell (ci, cj): nodes as (di, dj) offsets from its lower-left corner
    int d[3][2];
    if (((ci + cj) & 1) == 0) {
      if (sub == 0) { d[0][0] = 0; d[0][1] = 0; d[1][0] = 1; d[1][1] = 0; d[2][0] = 1; d[2][1] = 1; }
      else          { d[0][0] = 0; d[0][1] = 0; d[1][0] = 1; d[1][1] = 1; d[2][0] = 0; d[2][1] = 1; }
    } else {
      if (sub == 0) { d[0][0] = 0; d[0][1] = 0; d[1][0] = 1; d[1][1] = 0; d[2][0] = 0; d[2][1] = 1; }
      else          { d[0][0] = 1; d[0][1] = 0; d[1][0] = 1; d[1][1] = 1; d[2][0] = 0; d[2][1] = 1; }
    }
    double x[3][2], u[3][2], g[3][2], J;
#pragma unroll
    for (int n = 0; n < 3; ++n) {
      const int ln = (cy + d[n][1]) * kTileNX + cx + d[n][0];
      const double2 xn = xs[ln], un = us[ln];
      x[n][0] = xn.x; x[n][1] = xn.y;
      u[n][0] = un.x; u[n][1] = un.y;
    }
    simplex_geom<2, double>(x, g, &J);
    const double w = J * tri4_wsum();
    double eps[NV] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int n = 0; n < 3; ++n) add_strain<2, double>(g[n], u[n], eps);
    if (P.subscale) {
#pragma unroll
      for (int v = 0; v < NV; ++v) eps[v] += P.eps_macro[v];
    }
    const int m = __ldg(&P.emat[2 * (cj * gi.nx + ci) + sub]);
    double dd[ND];
    iso_from<2, double>(P.D[m], dd);
    double sig[NV];
    lei_stress_iso<2, double>(dd, eps, sig);
#pragma unroll
    for (int n = 0; n < 3; ++n) rec2[n * RN + k] = make_double2(g[n][0], g[n][1]);
    rec2[3 * RN + k] = make_double2(w, sig[0]);
    rec2[4 * RN + k] = make_double2(sig[1], sig[2]);
    recm[k] = (double)m;
  }
  __syncthreads();
  // C: row q of this thread's node (node entry t % 128: class 0 then class 1); one accumulator
  // serves both classes (class 1 uses its first 5 slots)
  const int q = t & 1;
  const int4 v = __ldg(&tnodes[t >> 1]);
  double acc[JAC ? Tri3Stencil0::NN : 1][2];
  const bool cls0 = (t >> 1) < kTileOwn / 2;
  if (v.x >= 0) {
    const int i = v.x % sx, j = v.x / sx;
    auto rows = [&](auto S) {
      using Sc = decltype(S);
      if constexpr (JAC) {
#pragma unroll
        for (int s = 0; s < Sc::NN; ++s) { acc[s][0] = 0.0; acc[s][1] = 0.0; }
      }
      double rr = 0.0;
#pragma unroll
      for (int a = 0; a < Sc::NADJ; ++a) {
        const int cx = i + Sc::ent(a, 0) - (i0 - 1), cy = j + Sc::ent(a, 1) - (j0 - 1);
        const int k = tile2_slot(cx, cy, Sc::ent(a, 3));
        double g[3][2];
#pragma unroll
        for (int n = 0; n < 3; ++n) { const double2 gn = rec2[n * RN + k]; g[n][0] = gn.x; g[n][1] = gn.y; }
        const double2 ws = rec2[3 * RN + k], s12 = rec2[4 * RN + k];
        const double w = ws.x;
        const double sig[NV] = {ws.y, s12.x, s12.y};
        const int la = Sc::ent(a, 4);
        rr += w * bt_sig<2, double>(g[la], sig, q);
        if constexpr (JAC) {
          const int m = (int)recm[k];
          T gk[3][2];
#pragma unroll
          for (int n = 0; n < 3; ++n) { gk[n][0] = (T)g[n][0]; gk[n][1] = (T)g[n][1]; }
          const T wk = (T)w;
          T dk[ND];
          if constexpr (sizeof(T) == sizeof(double)) iso_from<2, T>(P.D[m], dk);
          else iso_from<2, T>(P.Df[m], dk);
          T part[NV];
          part_iso<2, T>(dk, gk[la], q, part);
#pragma unroll
          for (int lb = 0; lb < 3; ++lb)
#pragma unroll
            for (int q2 = 0; q2 < 2; ++q2) acc[Sc::ent(a, 5 + lb)][q2] += (double)(wk * part_b<2, T>(part, gk[lb], q2));
        }
      }
      if (P.flags & FLAG_FUNC) P.Pf[v.y + q] = rr;
    };
    if (cls0) rows(Tri3Stencil0{});
    else rows(Tri3Stencil1{});
  }
  if constexpr (!JAC) return;
  if (!(P.flags & FLAG_JAC)) return;   // uniform over the CTA
  __syncthreads();   // the records are consumed: the stage takes their place
  double* stage = rec;
  if (v.x >= 0) {
    // the node's two rows, NN neighbour blocks each: [q][slot][d], one run of the CSR; stage
    // word a lives at tile2_swizzle(a)
    const int nn = cls0 ? Tri3Stencil0::NN : Tri3Stencil1::NN;
    const int o = v.w + q * nn * 2;
#pragma unroll
    for (int s = 0; s < Tri3Stencil0::NN; ++s)
      if (s < nn) { stage[tile2_swizzle(o + s * 2)] = acc[s][0]; stage[tile2_swizzle(o + s * 2 + 1)] = acc[s][1]; }
  }
  __syncthreads();
  // D: contiguous segments, a warp per segment
  const int lane = t & 31, warp = t >> 5;
  for (int sg = warp; sg < td.w; sg += kTileThreads / 32) {
    const int4 seg = __ldg(&segs[td.z + sg]);
    double* dst = P.val[0] + seg.y;
    for (int k = lane; k < seg.z; k += 32) dst[k] = stage[tile2_swizzle(seg.x + k)];
  }
}

// One CTA per tile.
template <typename T, bool JAC = true>
__global__ void __launch_bounds__(kTileThreads, 4) k_rows_tile2(DevProblem P, GridInfo gi, const int4* __restrict__ tiles,
                                                            const int4* __restrict__ tnodes, const int4* __restrict__ segs) {
  extern __shared__ double sm[];
  stencil_tile2<T, JAC>(P, gi, __ldg(&tiles[blockIdx.x]), tnodes + (size_t)blockIdx.x * kTileOwn, segs, sm);
}

// ------------------------------------------------------------------ 3D
constexpr int kT3 = 4;                                    // grid nodes per tile edge
constexpr int kT3N = kT3 + 2;                             // nodes with the halo, per edge
constexpr int kT3NodeN = kT3N * kT3N * kT3N;              // 216
constexpr int kT3C = kT3 + 1;                             // cells touching the tile, per edge
constexpr int kT3Cells = kT3C * kT3C * kT3C;              // 125
constexpr int kT3Elems = 6 * kT3Cells;                    // 750 tet4
constexpr int kT3Fields = 16;                             // g of nodes 1-3 (9), w, sigma (6)
constexpr int kT3Nodes = kT3 * kT3 * kT3;                 // 64
constexpr int kT3Threads = 3 * kT3Nodes;                  // a thread per node and row
constexpr int kT3Run = 3 * Tet4Stencil0::NN * 3;          // a node's three rows: 135 values

__host__ __device__ constexpr size_t tile3_smem_bytes() {
  // node data (x, u as six arrays), the record fields, the tet materials (bytes); the stage
  // reuses the record area
  return (size_t)(6 * kT3NodeN + kT3Fields * kT3Elems) * sizeof(double) + kT3Elems;
}
static_assert(kT3Fields * kT3Elems >= kT3Nodes * kT3Run, "the 3D stage fits the record area");

// Tet tt of the hex split of cell (i, j, k): its nodes as (di, dj, dk) corner offsets, in the
// connectivity order of the grid (corners n0 (0,0,0), n1 (1,0,0), n2 (1,1,0), n3 (0,1,0),
// n4 (0,0,1), n5 (1,0,1), n6 (1,1,1), n7 (0,1,1); tets {n0 n2 n3 n6}, {n0 n3 n7 n6},
// {n0 n7 n4 n6}, {n0 n5 n6 n4}, {n1 n5 n6 n0}, {n1 n6 n2 n0}).
__device__ __forceinline__ int tet_corner(int tt, int n) {
  constexpr unsigned char c[6][4] = {{0, 2, 3, 6}, {0, 3, 7, 6}, {0, 7, 4, 6}, {0, 5, 6, 4}, {1, 5, 6, 0}, {1, 6, 2, 0}};
  return c[tt][n];
}
__device__ __forceinline__ void corner_offset(int cn, int* o) {
  o[0] = (cn == 1 || cn == 2 || cn == 5 || cn == 6) ? 1 : 0;
  o[1] = (cn == 2 || cn == 3 || cn == 6 || cn == 7) ? 1 : 0;
  o[2] = (cn >= 4) ? 1 : 0;
}
// Record slot of tet tt of tile cell (cx, cy, cz): x fastest, so the node-row warps (consecutive
// nodes in x) read consecutive slots.
__host__ __device__ constexpr int tile3_slot(int cx, int cy, int cz, int tt) {
  return ((tt * kT3C + cz) * kT3C + cy) * kT3C + cx;
}

// Tile descriptor: two int4, {i0, j0, k0, 0} and {first segment, segment count, 0, 0}; per node
// (x fastest) an entry {node id or -1, first free DOF, first CSR slot, stage offset}; segments as
// in 2D.  Every thread of the CTA calls it.
template <typename T, bool JAC>
__device__ __forceinline__ void stencil_tile3(const DevProblem& P, const GridInfo& gi, int4 td, int4 ts,
                                              const int4* __restrict__ tnodes, const int4* __restrict__ segs,
                                              double* sm) {
  constexpr int NV = 6, ND = 12, NN = Tet4Stencil0::NN;
  constexpr int RN = kT3Elems;
  const int t = threadIdx.x;
  const int i0 = td.x, j0 = td.y, k0 = td.z;
  const int sx = gi.nx + 1, sxy = sx * (gi.ny + 1);
  double* xn = sm;                                           // x_d of node n at xn[d * kT3NodeN + n]
  double* un = sm + 3 * kT3NodeN;
  double* rec = sm + 6 * kT3NodeN;                           // field f of slot k at rec[f * RN + k]
  unsigned char* mat = reinterpret_cast<unsigned char*>(rec + kT3Fields * RN);
  // A: nodes
  for (int n = t; n < kT3NodeN; n += kT3Threads) {
    const int i = i0 - 1 + n % kT3N, j = j0 - 1 + (n / kT3N) % kT3N, k = k0 - 1 + n / (kT3N * kT3N);
    if (i >= 0 && i <= gi.nx && j >= 0 && j <= gi.ny && k >= 0 && k <= gi.nz) {
      const size_t id = (size_t)k * sxy + (size_t)j * sx + i;
#pragma unroll
      for (int d = 0; d < 3; ++d) { xn[d * kT3NodeN + n] = __ldg(&P.X[id * 3 + d]); un[d * kT3NodeN + n] = __ldg(&P.U[id * 3 + d]); }
    }
  }
  __syncthreads();
  // B: tets of the cells touching the tile, slot order
  for (int k = t; k < RN; k += kT3Threads) {
    const int cx = k % kT3C, cy = (k / kT3C) % kT3C, cz = (k / (kT3C * kT3C)) % kT3C, tt = k / kT3Cells;
    const int ci = i0 - 1 + cx, cj = j0 - 1 + cy, ck = k0 - 1 + cz;
    if (ci < 0 || ci >= gi.nx || cj < 0 || cj >= gi.ny || ck < 0 || ck >= gi.nz) continue;
    double x[4][3], u[4][3], g[4][3], J;
#pragma unroll
    for (int n = 0; n < 4; ++n) {
      int o[3];
      corner_offset(tet_corner(tt, n), o);
      const int ln = ((cz + o[2]) * kT3N + cy + o[1]) * kT3N + cx + o[0];
#pragma unroll
      for (int d = 0; d < 3; ++d) { x[n][d] = xn[d * kT3NodeN + ln]; u[n][d] = un[d * kT3NodeN + ln]; }
    }
    simplex_geom<3, double>(x, g, &J);
    const double w = J * tet5_wsum();
    double eps[NV] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int n = 0; n < 4; ++n) add_strain<3, double>(g[n], u[n], eps);
    if (P.subscale) {
#pragma unroll
      for (int v = 0; v < NV; ++v) eps[v] += P.eps_macro[v];
    }
    const int m = __ldg(&P.emat[6 * (((size_t)ck * gi.ny + cj) * gi.nx + ci) + tt]);
    double dd[ND];
    iso_from<3, double>(P.D[m], dd);
    double sig[NV];
    lei_stress_iso<3, double>(dd, eps, sig);
#pragma unroll
    for (int n = 1; n < 4; ++n)
#pragma unroll
      for (int d = 0; d < 3; ++d) rec[(3 * (n - 1) + d) * RN + k] = g[n][d];
    rec[9 * RN + k] = w;
#pragma unroll
    for (int v = 0; v < NV; ++v) rec[(10 + v) * RN + k] = sig[v];
    mat[k] = (unsigned char)m;
  }
  __syncthreads();
  // C: row q of node nl (warps 0-1 row 0, 2-3 row 1, 4-5 row 2: the row-dependent operations
  // stay uniform over a warp)
  const int nl = t % kT3Nodes, q = t / kT3Nodes;
  const int4 v = __ldg(&tnodes[nl]);
  double acc[JAC ? NN : 1][3];
  if (v.x >= 0) {
    using S = Tet4Stencil0;
    const int i = v.x % sx, j = (v.x / sx) % (gi.ny + 1), k = v.x / sxy;
    if constexpr (JAC) {
#pragma unroll
      for (int s = 0; s < NN; ++s) { acc[s][0] = 0.0; acc[s][1] = 0.0; acc[s][2] = 0.0; }
    }
    double rr = 0.0;
#pragma unroll
    for (int a = 0; a < S::NADJ; ++a) {
      const int cx = i + S::ent(a, 0) - (i0 - 1), cy = j + S::ent(a, 1) - (j0 - 1), cz = k + S::ent(a, 2) - (k0 - 1);
      const int el = tile3_slot(cx, cy, cz, S::ent(a, 3));
      double g[4][3];
#pragma unroll
      for (int n = 1; n < 4; ++n)
#pragma unroll
        for (int d = 0; d < 3; ++d) g[n][d] = rec[(3 * (n - 1) + d) * RN + el];
#pragma unroll
      for (int d = 0; d < 3; ++d) g[0][d] = -(g[1][d] + g[2][d] + g[3][d]);
      const double w = rec[9 * RN + el];
      double sig[NV];
#pragma unroll
      for (int vv = 0; vv < NV; ++vv) sig[vv] = rec[(10 + vv) * RN + el];
      const int la = S::ent(a, 4);
      rr += w * bt_sig<3, double>(g[la], sig, q);
      if constexpr (JAC) {
        const int m = mat[el];
        T gk[4][3];
#pragma unroll
        for (int n = 0; n < 4; ++n)
#pragma unroll
          for (int d = 0; d < 3; ++d) gk[n][d] = (T)g[n][d];
        const T wk = (T)w;
        T dk[ND];
        if constexpr (sizeof(T) == sizeof(double)) iso_from<3, T>(P.D[m], dk);
        else iso_from<3, T>(P.Df[m], dk);
        T part[NV];
        part_iso<3, T>(dk, gk[la], q, part);
#pragma unroll
        for (int lb = 0; lb < 4; ++lb)
#pragma unroll
          for (int q2 = 0; q2 < 3; ++q2) acc[S::ent(a, 5 + lb)][q2] += (double)(wk * part_b<3, T>(part, gk[lb], q2));
      }
    }
    if (P.flags & FLAG_FUNC) P.Pf[v.y + q] = rr;
  }
  if constexpr (!JAC) return;
  if (!(P.flags & FLAG_JAC)) return;   // uniform over the CTA
  __syncthreads();   // the records are consumed: the stage takes their place
  double* stage = rec;
  if (v.x >= 0) {
    double* o = stage + v.w + q * NN * 3;
#pragma unroll
    for (int s = 0; s < NN; ++s) { o[3 * s] = acc[s][0]; o[3 * s + 1] = acc[s][1]; o[3 * s + 2] = acc[s][2]; }
  }
  __syncthreads();
  // D: contiguous segments, a warp per segment
  const int lane = t & 31, warp = t >> 5;
  for (int sg = warp; sg < ts.y; sg += kT3Threads / 32) {
    const int4 seg = __ldg(&segs[ts.x + sg]);
    const double* src = stage + seg.x;
    double* dst = P.val[0] + seg.y;
    for (int kk = lane; kk < seg.z; kk += 32) dst[kk] = src[kk];
  }
}

// One CTA per 3D tile; tiles hold two int4 each ({i0, j0, k0, 0}, {first segment, segments, 0, 0}).
template <typename T, bool JAC = true>
__global__ void __launch_bounds__(kT3Threads) k_rows_tile3(DevProblem P, GridInfo gi, const int4* __restrict__ tiles,
                                                          const int4* __restrict__ tnodes, const int4* __restrict__ segs) {
  extern __shared__ double sm[];
  stencil_tile3<T, JAC>(P, gi, __ldg(&tiles[2 * blockIdx.x]), __ldg(&tiles[2 * blockIdx.x + 1]),
                        tnodes + (size_t)blockIdx.x * kT3Nodes, segs, sm);
}

}  // namespace pgd
