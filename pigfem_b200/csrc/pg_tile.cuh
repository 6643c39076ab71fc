// pg_tile.cuh -- tiled structured-grid rows: each element is formed once per tile.
//
// 2D (stencil_tile2).  The stencil nodes of a structured tri3 grid (pg_stencil.cuh) are grouped
// into tiles of 16 x 8 grid nodes.  One CTA of 256 threads takes a tile:
//   A. the coordinates and displacements of the tile's nodes and of a one-node halo (18 x 10)
//      go to shared memory;
//   B. every element of the 17 x 9 cells touching the tile (306 tri3) is formed once from them --
//      gradients, weight J W, stress -- into a shared record.  The element's nodes follow the
//      grid's union-jack split (the set-up checked every stencil node's elements against it);
//   C. one thread per stencil node and row q (warps 0-3 row 0, warps 4-7 row 1; in each half the
//      64 nodes of class 0 (8 elements) in two warps and the 64 of class 1 (4 elements) in the
//      other two) sums its block row and residual entry in adjacency order -- the operations of
//      stencil_rows, with each element's stress read from its record and its shape's gradients,
//      weight and element matrix from the constants -- keeping the row in registers and writing
//      the residual entry;
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
constexpr int kTileFields = 4;                             // doubles per record slot: stress, material
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
// store writes one value of each of 16 same-class nodes' rows (runs 56 doubles apart, so without
// it they meet in 4 bank pairs: 4 wavefronts); with it every row store and every warp-wide read
// of a segment is free of conflicts (one wavefront per half-warp).
__host__ __device__ constexpr int tile2_swizzle(int a) { return a ^ ((a >> 4) & 3); }

__host__ __device__ constexpr size_t tile2_smem_bytes() {
  // the nodes' displacements (double2), then the record fields; the stage reuses the record area
  return (size_t)(2 * kTileNodes2 + (kTileFields * kTileRecN > kTileY * kTileRowStage ? kTileFields * kTileRecN
                                                                                         : kTileY * kTileRowStage)) *
         sizeof(double);
}
static_assert((kTileY * kTileRowStage) % 4 == 0, "the swizzle stays inside the stage");

// Nodes of shape s (2 x cell parity + element in the cell) as (di, dj) corner offsets of its cell:
// the union-jack split of generate_mesh (cells with even i + j split along (0,0)-(1,1)).
// The offsets are packed two bits per (shape, node) -- di at bit 2 (3 s + n), dj above it -- so a
// runtime shape needs no table in local memory.
__host__ __device__ constexpr int tile2_shape_node(int s, int n, int c) {
  // shapes 0-3: {(0,0) (1,0) (1,1)}, {(0,0) (1,1) (0,1)}, {(0,0) (1,0) (0,1)}, {(1,0) (1,1) (0,1)}
  constexpr unsigned bits = (0u << 0) | (1u << 2) | (3u << 4) | (0u << 6) | (3u << 8) | (2u << 10) |
                            (0u << 12) | (1u << 14) | (2u << 16) | (1u << 18) | (3u << 20) | (2u << 22);
  return (int)((bits >> (2 * (3 * s + n) + c)) & 1u);
}
static_assert(tile2_shape_node(0, 2, 0) == 1 && tile2_shape_node(0, 2, 1) == 1 && tile2_shape_node(1, 2, 0) == 0 &&
              tile2_shape_node(1, 2, 1) == 1 && tile2_shape_node(3, 0, 0) == 1 && tile2_shape_node(3, 0, 1) == 0 &&
              tile2_shape_node(2, 1, 0) == 1 && tile2_shape_node(2, 2, 1) == 1, "shape offsets");

// The 2D tiles' strain, stress and internal-force arithmetic with every rounding explicit (no
// multiply-add contraction left to the compiler), so a tile's values do not depend on where the
// shape constants and D are read from: kernel parameters in a single launch, device memory in a
// batch.
__device__ __forceinline__ void t2_strain(const double* g, const double* u, double* e) {
  e[0] = __fma_rn(g[0], u[0], e[0]);
  e[1] = __fma_rn(g[1], u[1], e[1]);
  e[2] = __dadd_rn(e[2], __fma_rn(g[0], u[1], __dmul_rn(g[1], u[0])));
}
__device__ __forceinline__ void t2_stress(const double* d, const double* e, double* s) {
  s[0] = __fma_rn(d[1], e[1], __dmul_rn(d[0], e[0]));
  s[1] = __fma_rn(d[3], e[1], __dmul_rn(d[2], e[0]));
  s[2] = __dmul_rn(d[4], e[2]);
}
__device__ __forceinline__ double t2_bt_sig(const double* ga, const double* s, int q) {
  return (q == 0) ? __fma_rn(ga[1], s[2], __dmul_rn(ga[0], s[0])) : __fma_rn(ga[0], s[2], __dmul_rn(ga[1], s[1]));
}

// The shape constants of the 2D tiles (DevProblem::tile_*), one thread: the gradients and weight of
// each shape from the corners of the grid's first cell, and its element matrices per material
// from the element code (part_iso / part_b, as the per-element path forms them).  out: g (24), w
// (4), ke (432), kef (432, as doubles).
template <int DIM>
__global__ void k_tile2_consts(DevProblem P, double lo0, double lo1, double hx, double hy, double* out) {
  if constexpr (DIM == 2) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int sh = 0; sh < 4; ++sh) {
    double x[3][2], g[3][2], J;
    for (int n = 0; n < 3; ++n) {
      x[n][0] = __dadd_rn(lo0, __dmul_rn((double)tile2_shape_node(sh, n, 0), hx));
      x[n][1] = __dadd_rn(lo1, __dmul_rn((double)tile2_shape_node(sh, n, 1), hy));
    }
    simplex_geom<2, double>(x, g, &J);
    const double w = J * tri4_wsum();
    for (int n = 0; n < 3; ++n) { out[sh * 6 + n * 2] = g[n][0]; out[sh * 6 + n * 2 + 1] = g[n][1]; }
    out[24 + sh] = w;
    float gk[3][2];
    for (int n = 0; n < 3; ++n) { gk[n][0] = (float)g[n][0]; gk[n][1] = (float)g[n][1]; }
    const float wk = (float)w;
    for (int m = 0; m < 3; ++m) {
      double d[5];
      float df[5];
      iso_from<2, double>(P.D[m], d);
      iso_from<2, float>(P.Df[m], df);
      for (int la = 0; la < 3; ++la)
        for (int q = 0; q < 2; ++q) {
          double part[3];
          float partf[3];
          part_iso<2, double>(d, g[la], q, part);
          part_iso<2, float>(df, gk[la], q, partf);
          for (int lb = 0; lb < 3; ++lb)
            for (int q2 = 0; q2 < 2; ++q2) {
              const int i = (la * 2 + q) * 6 + lb * 2 + q2;
              out[28 + (sh * 3 + m) * 36 + i] = w * part_b<2, double>(part, g[lb], q2);
              out[28 + 432 + (sh * 3 + m) * 36 + i] = (double)(wk * part_b<2, float>(partf, gk[lb], q2));
            }
        }
    }
  }
  }
}

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
  // shared memory as double2 pairs, so each pair is one 16-byte access: the displacements of the
  // tile's nodes, then per record slot k the element's stress and material -- (sigma_xx,
  // sigma_yy) at rec2[k], (sigma_xy, material) at rec2[RN + k]
  double2* us = reinterpret_cast<double2*>(sm);
  double2* rec2 = us + kTileNodes2;
  double* rec = reinterpret_cast<double*>(rec2);       // the stage, after the records are consumed
  // A: nodes
  for (int k = t; k < kTileNodes2; k += kTileThreads) {
    const int i = i0 - 1 + k % kTileNX, j = j0 - 1 + k / kTileNX;
    if (i >= 0 && i <= gi.nx && j >= 0 && j <= gi.ny) us[k] = __ldg(reinterpret_cast<const double2*>(P.U) + j * sx + i);
  }
  __syncthreads();
  // B: elements of the cells touching the tile, cell order (consecutive lanes read consecutive
  // nodes): strain and stress into the element's record slot; the gradients are the shape's
  for (int it = t; it < 2 * kTileCX * kTileCY; it += kTileThreads) {
    const int cx = it % kTileCX, cy = (it / kTileCX) % kTileCY, sub = it / (kTileCX * kTileCY);
    const int k = tile2_slot(cx, cy, sub);
    const int ci = i0 - 1 + cx, cj = j0 - 1 + cy;
    if (ci < 0 || ci >= gi.nx || cj < 0 || cj >= gi.ny) continue;
    const int sh = 2 * ((ci + cj) & 1) + sub;
    double eps[NV] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int n = 0; n < 3; ++n) {
      const double2 un = us[(cy + tile2_shape_node(sh, n, 1)) * kTileNX + cx + tile2_shape_node(sh, n, 0)];
      const double u[2] = {un.x, un.y};
      t2_strain(P.tile_g[sh][n], u, eps);
    }
    if (P.subscale) {
#pragma unroll
      for (int v = 0; v < NV; ++v) eps[v] = __dadd_rn(eps[v], P.eps_macro[v]);
    }
    const int m = __ldg(&P.emat[2 * (cj * gi.nx + ci) + sub]);
    double dd[ND];
    iso_from<2, double>(P.D[m], dd);
    double sig[NV];
    t2_stress(dd, eps, sig);
    rec2[k] = make_double2(sig[0], sig[1]);
    rec2[RN + k] = make_double2(sig[2], (double)m);
  }
  __syncthreads();
  // C: row q of this thread's node (warps 0-3 row 0, 4-7 row 1; node entry t % 128: class 0 then
  // class 1, so a warp's nodes share a class); one accumulator serves both classes (class 1 uses
  // its first 5 slots).  Per adjacent element: its stress and material from the record, its
  // shape's gradients, weight and element matrix from the constants (the shape follows from the
  // node's class and the element's place in the stencil; with the row uniform over a warp the
  // element-matrix reads are broadcasts from the constant bank)
  const int q = t / kTileOwn;
  const int4 v = __ldg(&tnodes[t % kTileOwn]);
  double acc[JAC ? Tri3Stencil0::NN : 1][2];
  const bool cls0 = (t % kTileOwn) < kTileOwn / 2;
  if (v.x >= 0) {
    const int i = v.x % sx, j = v.x / sx;
    auto rows = [&](auto S) {
      using Sc = decltype(S);
      constexpr int CLS = (Sc::NN == Tri3Stencil0::NN) ? 0 : 1;
      if constexpr (JAC) {
#pragma unroll
        for (int s = 0; s < Sc::NN; ++s) { acc[s][0] = 0.0; acc[s][1] = 0.0; }
      }
      double rr = 0.0;
#pragma unroll
      for (int a = 0; a < Sc::NADJ; ++a) {
        const int cx = i + Sc::ent(a, 0) - (i0 - 1), cy = j + Sc::ent(a, 1) - (j0 - 1);
        const int k = tile2_slot(cx, cy, Sc::ent(a, 3));
        const int sh = 2 * ((CLS + Sc::ent(a, 0) + Sc::ent(a, 1)) & 1) + Sc::ent(a, 3);
        const int la = Sc::ent(a, 4);
        const double2 s01 = rec2[k], s2m = rec2[RN + k];
        const double sig[NV] = {s01.x, s01.y, s2m.x};
        rr = __fma_rn(P.tile_w[sh], t2_bt_sig(P.tile_g[sh][la], sig, q), rr);
        if constexpr (JAC) {
          const int m = (int)s2m.y;
          const int row = (la * 2 + q) * 6;
#pragma unroll
          for (int lb = 0; lb < 3; ++lb)
#pragma unroll
            for (int q2 = 0; q2 < 2; ++q2) {
              const double kv = (sizeof(T) == sizeof(double)) ? P.tile_ke[sh][m][row + lb * 2 + q2]
                                                              : (double)P.tile_kef[sh][m][row + lb * 2 + q2];
              acc[Sc::ent(a, 5 + lb)][q2] = __dadd_rn(acc[Sc::ent(a, 5 + lb)][q2], kv);
            }
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
constexpr int kT3Fields = 6;                              // the element's stress (6); its material in mat[]
constexpr int kT3Nodes = kT3 * kT3 * kT3;                 // 64
constexpr int kT3Threads = 3 * kT3Nodes;                  // a thread per node and row
constexpr int kT3Run = 3 * Tet4Stencil0::NN * 3;          // a node's three rows: 135 values

constexpr int kT3Area = (kT3Fields * kT3Elems > kT3Nodes * kT3Run) ? kT3Fields * kT3Elems : kT3Nodes * kT3Run;
__host__ __device__ constexpr size_t tile3_smem_bytes() {
  // the nodes' displacements (three arrays), the record fields (the stage reuses their area),
  // the tet materials (bytes)
  return (size_t)(3 * kT3NodeN + kT3Area) * sizeof(double) + kT3Elems;
}

// Every uncut tet of the uniform hex grid is one of six shapes, the tet's place in the hex split
// (the same in every cell): per shape the gradients of its four nodes, its weight J W and its
// element matrix per bulk material ([(la * 3 + q) * 12 + lb * 3 + q2]), formed once at upload by
// the element code (k_tile3_consts).  A single launch takes them as a kernel parameter, a batch
// from device memory.
struct Tile3Const {
  double g[6][4][3];
  double w[6];
  double ke[6][3][144];
};

// The 3D tiles' arithmetic with every rounding explicit (see t2_strain).
__device__ __forceinline__ void t3_strain(const double* g, const double* u, double* e) {
  e[0] = __fma_rn(g[0], u[0], e[0]);
  e[1] = __fma_rn(g[1], u[1], e[1]);
  e[2] = __fma_rn(g[2], u[2], e[2]);
  e[3] = __dadd_rn(e[3], __fma_rn(g[1], u[2], __dmul_rn(g[2], u[1])));
  e[4] = __dadd_rn(e[4], __fma_rn(g[0], u[2], __dmul_rn(g[2], u[0])));
  e[5] = __dadd_rn(e[5], __fma_rn(g[0], u[1], __dmul_rn(g[1], u[0])));
}
__device__ __forceinline__ void t3_stress(const double* d, const double* e, double* s) {
  s[0] = __fma_rn(d[2], e[2], __fma_rn(d[1], e[1], __dmul_rn(d[0], e[0])));
  s[1] = __fma_rn(d[5], e[2], __fma_rn(d[4], e[1], __dmul_rn(d[3], e[0])));
  s[2] = __fma_rn(d[8], e[2], __fma_rn(d[7], e[1], __dmul_rn(d[6], e[0])));
  s[3] = __dmul_rn(d[9], e[3]);
  s[4] = __dmul_rn(d[10], e[4]);
  s[5] = __dmul_rn(d[11], e[5]);
}
__device__ __forceinline__ double t3_bt_sig(const double* ga, const double* s, int q) {
  if (q == 0) return __fma_rn(ga[1], s[5], __fma_rn(ga[2], s[4], __dmul_rn(ga[0], s[0])));
  if (q == 1) return __fma_rn(ga[0], s[5], __fma_rn(ga[2], s[3], __dmul_rn(ga[1], s[1])));
  return __fma_rn(ga[0], s[4], __fma_rn(ga[1], s[3], __dmul_rn(ga[2], s[2])));
}

// Tet tt of the hex split of cell (i, j, k): its nodes as (di, dj, dk) corner offsets, in the
// connectivity order of the grid (corners n0 (0,0,0), n1 (1,0,0), n2 (1,1,0), n3 (0,1,0),
// n4 (0,0,1), n5 (1,0,1), n6 (1,1,1), n7 (0,1,1); tets {n0 n2 n3 n6}, {n0 n3 n7 n6},
// {n0 n7 n4 n6}, {n0 n5 n6 n4}, {n1 n5 n6 n0}, {n1 n6 n2 n0}).
// (packed a nibble per corner, 16 bits per tet, so a runtime tet index needs no table in local
// memory)
__host__ __device__ constexpr int tet_corner(int tt, int n) {
  constexpr unsigned long long lo = 0x4650647067306320ull;   // tets 0-3
  constexpr unsigned hi = 0x02610651u;                      // tets 4-5
  return (int)(((tt < 4 ? (lo >> (16 * tt)) : (unsigned long long)(hi >> (16 * (tt - 4)))) >> (4 * n)) & 15u);
}
static_assert(tet_corner(0, 1) == 2 && tet_corner(1, 2) == 7 && tet_corner(2, 2) == 4 && tet_corner(3, 1) == 5 &&
              tet_corner(4, 0) == 1 && tet_corner(4, 3) == 0 && tet_corner(5, 2) == 2 && tet_corner(5, 1) == 6 &&
              tet_corner(3, 3) == 4 && tet_corner(0, 3) == 6, "tet corners");
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

// The shape constants of the 3D tiles, one thread: the gradients and weight of each tet of the
// grid's first cell from its corners, and its element matrices per material from the element code.
template <int DIM>
__global__ void k_tile3_consts(DevProblem P, double lo0, double lo1, double lo2, double hx, double hy, double hz,
                               Tile3Const* out) {
  if constexpr (DIM == 3) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double lo[3] = {lo0, lo1, lo2}, h[3] = {hx, hy, hz};
  for (int tt = 0; tt < 6; ++tt) {
    double x[4][3], g[4][3], J;
    for (int n = 0; n < 4; ++n) {
      int o[3];
      corner_offset(tet_corner(tt, n), o);
      for (int d = 0; d < 3; ++d) x[n][d] = __dadd_rn(lo[d], __dmul_rn((double)o[d], h[d]));
    }
    simplex_geom<3, double>(x, g, &J);
    const double w = J * tet5_wsum();
    for (int n = 0; n < 4; ++n) for (int d = 0; d < 3; ++d) out->g[tt][n][d] = g[n][d];
    out->w[tt] = w;
    for (int m = 0; m < 3; ++m) {
      double dd[12];
      iso_from<3, double>(P.D[m], dd);
      for (int la = 0; la < 4; ++la)
        for (int q = 0; q < 3; ++q) {
          double part[6];
          part_iso<3, double>(dd, g[la], q, part);
          for (int lb = 0; lb < 4; ++lb)
            for (int q2 = 0; q2 < 3; ++q2) out->ke[tt][m][(la * 3 + q) * 12 + lb * 3 + q2] = w * part_b<3, double>(part, g[lb], q2);
        }
    }
  }
  }
}

// Tile descriptor: two int4, {i0, j0, k0, 0} and {first segment, segment count, 0, 0}; per node
// (x fastest) an entry {node id or -1, first free DOF, first CSR slot, stage offset}; segments as
// in 2D.  Every thread of the CTA calls it.
template <typename T, bool JAC>
__device__ __forceinline__ void stencil_tile3(const DevProblem& P, const GridInfo& gi, int4 td, int4 ts,
                                              const int4* __restrict__ tnodes, const int4* __restrict__ segs,
                                              double* sm, const Tile3Const& C) {
  constexpr int NV = 6, ND = 12, NN = Tet4Stencil0::NN;
  constexpr int RN = kT3Elems;
  const int t = threadIdx.x;
  const int i0 = td.x, j0 = td.y, k0 = td.z;
  const int sx = gi.nx + 1, sxy = sx * (gi.ny + 1);
  double* un = sm;                                           // u_d of node n at un[d * kT3NodeN + n]
  double* rec = sm + 3 * kT3NodeN;                           // stress component f of slot k at rec[f * RN + k]
  unsigned char* mat = reinterpret_cast<unsigned char*>(rec + kT3Area);
  // A: nodes
  for (int n = t; n < kT3NodeN; n += kT3Threads) {
    const int i = i0 - 1 + n % kT3N, j = j0 - 1 + (n / kT3N) % kT3N, k = k0 - 1 + n / (kT3N * kT3N);
    if (i >= 0 && i <= gi.nx && j >= 0 && j <= gi.ny && k >= 0 && k <= gi.nz) {
      const size_t id = (size_t)k * sxy + (size_t)j * sx + i;
#pragma unroll
      for (int d = 0; d < 3; ++d) un[d * kT3NodeN + n] = __ldg(&P.U[id * 3 + d]);
    }
  }
  __syncthreads();
  // B: tets of the cells touching the tile, slot order: strain and stress into the record (the
  // gradients are the shape's)
  for (int k = t; k < RN; k += kT3Threads) {
    const int cx = k % kT3C, cy = (k / kT3C) % kT3C, cz = (k / (kT3C * kT3C)) % kT3C, tt = k / kT3Cells;
    const int ci = i0 - 1 + cx, cj = j0 - 1 + cy, ck = k0 - 1 + cz;
    if (ci < 0 || ci >= gi.nx || cj < 0 || cj >= gi.ny || ck < 0 || ck >= gi.nz) continue;
    double eps[NV] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int n = 0; n < 4; ++n) {
      int o[3];
      corner_offset(tet_corner(tt, n), o);
      const int ln = ((cz + o[2]) * kT3N + cy + o[1]) * kT3N + cx + o[0];
      const double u[3] = {un[ln], un[kT3NodeN + ln], un[2 * kT3NodeN + ln]};
      t3_strain(C.g[tt][n], u, eps);
    }
    if (P.subscale) {
#pragma unroll
      for (int v = 0; v < NV; ++v) eps[v] = __dadd_rn(eps[v], P.eps_macro[v]);
    }
    const int m = __ldg(&P.emat[6 * (((size_t)ck * gi.ny + cj) * gi.nx + ci) + tt]);
    double dd[ND];
    iso_from<3, double>(P.D[m], dd);
    double sig[NV];
    t3_stress(dd, eps, sig);
#pragma unroll
    for (int v = 0; v < NV; ++v) rec[v * RN + k] = sig[v];
    mat[k] = (unsigned char)m;
  }
  __syncthreads();
  // C: row q of node nl (warps 0-1 row 0, 2-3 row 1, 4-5 row 2: the row-dependent operations
  // stay uniform over a warp); per adjacent tet its stress and material from the record, its
  // shape's gradients, weight and element-matrix entries from the constants
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
      const int tt = S::ent(a, 3), la = S::ent(a, 4);
      const int el = tile3_slot(cx, cy, cz, tt);
      double sig[NV];
#pragma unroll
      for (int vv = 0; vv < NV; ++vv) sig[vv] = rec[vv * RN + el];
      rr = __fma_rn(C.w[tt], t3_bt_sig(C.g[tt][la], sig, q), rr);
      if constexpr (JAC) {
        const int m = mat[el];
        const double* kr = C.ke[tt][m] + (la * 3 + q) * 12;
#pragma unroll
        for (int lb = 0; lb < 4; ++lb)
#pragma unroll
          for (int q2 = 0; q2 < 3; ++q2) {
            const double kv = (sizeof(T) == sizeof(double)) ? kr[lb * 3 + q2] : (double)(float)kr[lb * 3 + q2];
            acc[S::ent(a, 5 + lb)][q2] = __dadd_rn(acc[S::ent(a, 5 + lb)][q2], kv);
          }
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
                                                          const int4* __restrict__ tnodes, const int4* __restrict__ segs,
                                                          Tile3Const C) {
  extern __shared__ double sm[];
  stencil_tile3<T, JAC>(P, gi, __ldg(&tiles[2 * blockIdx.x]), __ldg(&tiles[2 * blockIdx.x + 1]),
                        tnodes + (size_t)blockIdx.x * kT3Nodes, segs, sm, C);
}

}  // namespace pgd
