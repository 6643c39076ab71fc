// pg_prep.cu -- IGFEM preprocessing on the device: the O(nodes x inclusions) and O(elements)
// passes of the set-up.
//
//   node detection      Mesh::detect_node (src/Mesh.cpp:2727-2929) with the circle and sphere
//                       tests (src/InclusionCircle.cpp:150-163, src/InclusionSphere.cpp): per
//                       standard node the last inclusion (in reverse order, the reference's loop)
//                       whose bounding box holds the node and whose level set is below -1e-12;
//                       a node within 1e-12 of a surface stops the set-up, as the reference does;
//   element pass        the all-equal test of the element detection (Tri3/Quad4/Tet4::detection):
//                       an element whose nodes share one value is uncut (inside a fiber when the
//                       value is an inclusion); the others are candidates for the cut-case tables;
//   cut edges           Mesh::add_enrichments (src/Mesh.cpp:3103-3252): the distinct (edge,
//                       inclusion) pairs of the cut elements, numbered in the order of the
//                       reference's std::set<(sorted node pair, inclusion)>, and the point where
//                       each edge meets its inclusion's surface (Inclusion::find_intersection,
//                       src/Inclusion.cpp:32-121: Steffensen from the midpoint, Brent fallback);
//   DOF numbering       DofObject::set_local_owned_normal_dofs (src/DofObject.cpp:336-385) for the
//                       standard nodes of the structured grid: free DOFs in node order, the
//                       constrained ones numbered apart, both in closed form from the node's grid
//                       position (the Dirichlet or periodic conditions of Tests/Main.cpp:549-581);
//   pattern             (device_pattern, at the end of this file) the DOF nodes' adjacency, their
//                       sorted neighbours and the four CSR patterns (Solver::preallocate_matrix,
//                       src/Solver.cpp:426-490, 772-896), from sorted 64-bit keys.
//
// This file is compiled without floating-point contraction (-fmad=false), so every coordinate,
// level-set value and root iterate is formed with the same IEEE operations, in the same order, as
// the host set-up (pg_setup.cpp): node tables and edge lists are bitwise those of the host, and
// the intersection points too.
//
// Cut edges are marked in a flag array over (node, edge direction, inclusion slot): from its lower
// node id every edge of the structured grids runs in one of 4 (2D) or 7 (3D) directions, listed in
// increasing id offset, and an edge between two inclusions carries two enrichment nodes (the lower
// inclusion first).  An exclusive scan of the flags is then the reference's set order.  The rule
// "an edge whose end nodes differ carries one enrichment node per inclusion among them" is the one
// every tri3 case follows; for quad4 and tet4 elements that see two inclusions the cut-case tables
// have their own cases, so there the host forms the edges from the tables instead.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "pg_roots.h"
#include "pg_setup.h"

namespace pgp {

struct Grid {
  int dim, etype, nx, ny, nz, ninc;
  double lo[3], h[3];
  const double* incl;   // device: circles (cx, cy, r) / spheres (cx, cy, cz, r)
};

constexpr int kDirs2 = 4, kDirs3 = 7;

// Coordinate of grid index i along axis q: lo + i h, as the host forms it.
__device__ __forceinline__ double grid_x(const Grid& g, int q, int i) { return g.lo[q] + (double)i * g.h[q]; }

__device__ __forceinline__ void node_xyz(const Grid& g, int id, double* x) {
  const int sx = g.nx + 1, sxy = sx * (g.ny + 1);
  const int i = id % sx, j = (id / sx) % (g.ny + 1), k = id / sxy;
  x[0] = grid_x(g, 0, i);
  x[1] = grid_x(g, 1, j);
  x[2] = (g.dim == 3) ? grid_x(g, 2, k) : 0.0;
}

// Circle / sphere of inclusion f: bounding box (the sphere's upper z bound is cy + r, as the
// reference writes it) and the detection value: 0 outside, 1 on the surface, 2 inside.
__device__ __forceinline__ int detect_one(const Grid& g, int f, const double* x) {
  if (g.dim == 2) {
    const double cx = g.incl[3 * f], cy = g.incl[3 * f + 1], r = g.incl[3 * f + 2];
    if (!((cx - r <= x[0]) && (cy - r <= x[1]) && (x[0] <= cx + r) && (x[1] <= cy + r))) return 0;
    const double dx = x[0] - cx, dy = x[1] - cy;
    const double val = (sqrt(dx * dx + dy * dy) - r) / r;
    return val > 1e-12 ? 0 : (val < -1e-12 ? 2 : 1);
  }
  const double cx = g.incl[4 * f], cy = g.incl[4 * f + 1], cz = g.incl[4 * f + 2], r = g.incl[4 * f + 3];
  if (!((cx - r <= x[0]) && (cy - r <= x[1]) && (cz - r <= x[2]) && (x[0] <= cx + r) && (x[1] <= cy + r) && (x[2] <= cy + r)))
    return 0;
  const double gx = (x[0] - cx) / r, gy = (x[1] - cy) / r, gz = (x[2] - cz) / r;
  const double val = gx * gx + gy * gy + gz * gz - 1.0;
  return val > 1e-12 ? 0 : (val < -1e-12 ? 2 : 1);
}

__global__ void k_prep_nodes(Grid g, int n_std, int* __restrict__ detect, int* __restrict__ surface_first) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= n_std) return;
  double x[3];
  node_xyz(g, id, x);
  int res = -1;
  for (int f = g.ninc - 1; f >= 0; --f) {
    const int r = detect_one(g, f, x);
    if (r == 0) continue;
    if (r == 1) { atomicMin(surface_first, id); res = -1; break; }
    res = f;
    break;
  }
  detect[id] = res;
}

// Nodes of element e of the structured grid, in the host's connectivity order.
__device__ __forceinline__ int elem_nodes(const Grid& g, int e, int* nd) {
  const int sx = g.nx + 1, sxy = sx * (g.ny + 1);
  if (g.etype == pg::TRI3) {
    const int cell = e >> 1, sub = e & 1;
    const int i = cell % g.nx, j = cell / g.nx;
    const int n00 = j * sx + i, n10 = n00 + 1, n01 = n00 + sx, n11 = n01 + 1;
    if (((i + j) & 1) == 0) {
      if (sub == 0) { nd[0] = n00; nd[1] = n10; nd[2] = n11; }
      else { nd[0] = n00; nd[1] = n11; nd[2] = n01; }
    } else {
      if (sub == 0) { nd[0] = n00; nd[1] = n10; nd[2] = n01; }
      else { nd[0] = n10; nd[1] = n11; nd[2] = n01; }
    }
    return 3;
  }
  if (g.etype == pg::QUAD4) {
    const int i = e % g.nx, j = e / g.nx;
    const int n00 = j * sx + i;
    nd[0] = n00; nd[1] = n00 + 1; nd[2] = n00 + sx + 1; nd[3] = n00 + sx;
    return 4;
  }
  const int hex = e / 6, t = e % 6;
  const int i = hex % g.nx, j = (hex / g.nx) % g.ny, k = hex / (g.nx * g.ny);
  const int n0 = k * sxy + j * sx + i;
  const int c[8] = {n0, n0 + 1, n0 + sx + 1, n0 + sx, n0 + sxy, n0 + sxy + 1, n0 + sxy + sx + 1, n0 + sxy + sx};
  constexpr unsigned char tets[6][4] = {{0, 2, 3, 6}, {0, 3, 7, 6}, {0, 7, 4, 6}, {0, 5, 6, 4}, {1, 5, 6, 0}, {1, 6, 2, 0}};
#pragma unroll
  for (int q = 0; q < 4; ++q) nd[q] = c[tets[t][q]];
  return 4;
}

// Direction code of the edge from node a to node b > a (offsets in increasing order; -1 if the
// offset is not an edge direction of the grid).
__device__ __forceinline__ int edge_dir(const Grid& g, int a, int b) {
  const int sx = g.nx + 1, sxy = sx * (g.ny + 1), o = b - a;
  if (g.dim == 2) {
    if (o == 1) return 0;
    if (o == sx - 1) return 1;
    if (o == sx) return 2;
    if (o == sx + 1) return 3;
    return -1;
  }
  const int offs[kDirs3] = {1, sx, sx + 1, sxy, sxy + 1, sxy + sx, sxy + sx + 1};
#pragma unroll
  for (int d = 0; d < kDirs3; ++d) if (o == offs[d]) return d;
  return -1;
}

// Element pass: flag 0 uncut with its own material, 1 inside inclusion (all nodes in one), 2 a
// candidate for the cut-case tables.  Candidates also mark their cut edges, unless the element
// sees two inclusions in a quad4 / tet4 mesh (then *rule_ok is cleared and the host forms edges).
__global__ void k_prep_elems(Grid g, int ne, const int* __restrict__ detect, unsigned char* __restrict__ flag,
                             unsigned char* __restrict__ emark, int* __restrict__ eincl, int* __restrict__ rule_ok,
                             int* __restrict__ bad_edge) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  int nd[4], v[4];
  const int npe = elem_nodes(g, e, nd);
  bool same = true;
  int n_incl = 0, first = -1;
  for (int q = 0; q < npe; ++q) {
    v[q] = detect[nd[q]];
    same &= v[q] == v[0];
  }
  if (same) { flag[e] = (v[0] != -1) ? 1 : 0; return; }
  flag[e] = 2;
  for (int q = 0; q < npe; ++q)
    if (v[q] >= 0 && v[q] != first) {
      if (first < 0) { first = v[q]; n_incl = 1; }
      else n_incl = 2;
    }
  if (g.etype != pg::TRI3 && n_incl > 1) { *rule_ok = 0; return; }
  const int ndir = (g.dim == 2) ? kDirs2 : kDirs3;
  constexpr unsigned char tri_e[3][2] = {{0, 1}, {1, 2}, {2, 0}};
  constexpr unsigned char quad_e[4][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}};
  constexpr unsigned char tet_e[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {1, 3}, {2, 3}};
  const int nedge = (g.etype == pg::TRI3) ? 3 : (g.etype == pg::QUAD4 ? 4 : 6);
  for (int k = 0; k < nedge; ++k) {
    const int p = (g.etype == pg::TRI3) ? tri_e[k][0] : (g.etype == pg::QUAD4 ? quad_e[k][0] : tet_e[k][0]);
    const int q = (g.etype == pg::TRI3) ? tri_e[k][1] : (g.etype == pg::QUAD4 ? quad_e[k][1] : tet_e[k][1]);
    if (v[p] == v[q]) continue;
    const int a = min(nd[p], nd[q]), b = max(nd[p], nd[q]);
    const int d = edge_dir(g, a, b);
    if (d < 0) { atomicExch(bad_edge, 1); continue; }
    const int lo = min(v[p], v[q]), hi = max(v[p], v[q]);
    const size_t base = ((size_t)a * ndir + d) * 2;
    if (lo < 0) { emark[base] = 1; eincl[base] = hi; }
    else { emark[base] = 1; eincl[base] = lo; emark[base + 1] = 1; eincl[base + 1] = hi; }
  }
}

// ------------------------------------------------------------------ exclusive scan of byte flags
constexpr int kScanThreads = 256, kScanItems = 8, kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ int block_exclusive(int v, int* sh, int* total) {
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) { const int y = __shfl_up_sync(0xffffffffu, x, o); if (lane >= o) x += y; }
  if (lane == 31) sh[w] = x;
  __syncthreads();
  if (w == 0) {
    int s = (lane < kScanThreads / 32) ? sh[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) { const int y = __shfl_up_sync(0xffffffffu, s, o); if (lane >= o) s += y; }
    if (lane < kScanThreads / 32) sh[lane] = s;
  }
  __syncthreads();
  const int before = (w > 0 ? sh[w - 1] : 0) + x - v;
  *total = sh[kScanThreads / 32 - 1];
  __syncthreads();
  return before;
}

__global__ void k_scan_count(const unsigned char* __restrict__ f, size_t n, int* __restrict__ tile_sum) {
  __shared__ int sh[kScanThreads / 32];
  const size_t base = (size_t)blockIdx.x * kScanTile + (size_t)threadIdx.x * kScanItems;
  int c = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) if (base + k < n) c += f[base + k] != 0;
  int total;
  block_exclusive(c, sh, &total);
  if (threadIdx.x == 0) tile_sum[blockIdx.x] = total;
}

// One block: exclusive scan of the tile sums in place (sequential over chunks of the block size).
__global__ void k_scan_tiles(int* __restrict__ tile_sum, int ntiles, int* __restrict__ grand) {
  __shared__ int sh[kScanThreads / 32];
  int carry = 0;
  for (int b = 0; b < ntiles; b += kScanThreads) {
    const int i = b + threadIdx.x;
    const int v = (i < ntiles) ? tile_sum[i] : 0;
    int total;
    const int ex = block_exclusive(v, sh, &total);
    if (i < ntiles) tile_sum[i] = carry + ex;
    carry += total;
  }
  if (threadIdx.x == 0) *grand = carry;
}

// Writes, for every set flag, its rank into idx (and the flagged position into list, if given).
__global__ void k_scan_write(const unsigned char* __restrict__ f, size_t n, const int* __restrict__ tile_sum,
                             int* __restrict__ idx, int* __restrict__ list) {
  __shared__ int sh[kScanThreads / 32];
  const size_t base = (size_t)blockIdx.x * kScanTile + (size_t)threadIdx.x * kScanItems;
  int c = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) if (base + k < n) c += f[base + k] != 0;
  int total;
  int r = tile_sum[blockIdx.x] + block_exclusive(c, sh, &total);
#pragma unroll
  for (int k = 0; k < kScanItems; ++k)
    if (base + k < n && f[base + k]) {
      if (idx) idx[base + k] = r;
      if (list) list[r] = (int)(base + k);
      ++r;
    }
}

// ------------------------------------------------------------------ enrichment nodes
struct EdgeFnDev {
  const Grid* g;
  int inc;
  double p0[3], p1[3];
  // level set along p0 -> p1 and its derivative (InclusionCircle::int_fdf / InclusionSphere)
  __device__ void eval(double a, double* f, double* df) const {
    if (g->dim == 2) {
      const double cx = g->incl[3 * inc], cy = g->incl[3 * inc + 1], r = g->incl[3 * inc + 2];
      const double g0 = p0[0] + a * (p1[0] - p0[0]) - cx;
      const double g1 = p0[1] + a * (p1[1] - p0[1]) - cy;
      const double d0 = p1[0] - p0[0], d1 = p1[1] - p0[1];
      const double s0 = g0 / r, s1 = g1 / r;
      *f = s0 * s0 + s1 * s1 - 1;
      *df = (1 / (r * r)) * 2.0 * (g0 * d0 + g1 * d1);
    } else {
      const double cx = g->incl[4 * inc], cy = g->incl[4 * inc + 1], cz = g->incl[4 * inc + 2], r = g->incl[4 * inc + 3];
      const double g0 = p0[0] + a * (p1[0] - p0[0]) - cx;
      const double g1 = p0[1] + a * (p1[1] - p0[1]) - cy;
      const double g2 = p0[2] + a * (p1[2] - p0[2]) - cz;
      const double d0 = p1[0] - p0[0], d1 = p1[1] - p0[1], d2 = p1[2] - p0[2];
      const double s0 = g0 / r, s1 = g1 / r, s2 = g2 / r;
      *f = s0 * s0 + s1 * s1 + s2 * s2 - 1.0;
      *df = (2.0 / (r * r)) * (g0 * d0 + g1 * d1 + g2 * d2);
    }
  }
};

// One thread per enrichment node k (flag position list[k] = (a * ndir + d) * 2 + slot).
__global__ void k_prep_roots(Grid g, int n_enr, const int* __restrict__ list, const int* __restrict__ eincl,
                             int* __restrict__ enr_edge, int* __restrict__ enr_incl, double* __restrict__ XE,
                             int* __restrict__ no_sign_change) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_enr) return;
  const int pos = list[k];
  const int ndir = (g.dim == 2) ? kDirs2 : kDirs3;
  const int a = pos / (2 * ndir), d = (pos / 2) % ndir;
  const int sx = g.nx + 1, sxy = sx * (g.ny + 1);
  int o;
  if (g.dim == 2) o = (d == 0) ? 1 : (d == 1 ? sx - 1 : (d == 2 ? sx : sx + 1));
  else {
    const int offs[kDirs3] = {1, sx, sx + 1, sxy, sxy + 1, sxy + sx, sxy + sx + 1};
    o = offs[d];
  }
  const int b = a + o, inc = eincl[pos];
  EdgeFnDev fn;
  fn.g = &g;
  fn.inc = inc;
  node_xyz(g, a, fn.p0);
  node_xyz(g, b, fn.p1);
  double fa, fb, dfa;
  fn.eval(0.0, &fa, &dfa);
  fn.eval(1.0, &fb, &dfa);
  if (fa * fb >= 0) atomicMin(no_sign_change, k);
  const double alpha = pg::steffensen_then_brent(fn);
#pragma unroll
  for (int q = 0; q < 3; ++q) XE[(size_t)k * 3 + q] = fn.p0[q] + alpha * (fn.p1[q] - fn.p0[q]);
  enr_edge[2 * k] = a;
  enr_edge[2 * k + 1] = b;
  enr_incl[k] = inc;
}

// ------------------------------------------------------------------ DOF numbering
// Standard node n, direction q: the free index among the standard nodes' free DOFs (>= 0), or
// -1 - p for the p-th constrained DOF; periodic images get their primary's numbers.
__global__ void k_prep_dofs(Grid g, int n_std, int subscale, int* __restrict__ dof) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= n_std) return;
  const int dim = g.dim;
  const int sx = g.nx + 1, sxy = sx * (g.ny + 1);
  const int i = n % sx, j = (n / sx) % (g.ny + 1), k = n / sxy;
  if (subscale) {
    // primaries: i < nx, j < ny (k < nz), numbered in id order; node 0 is pinned
    const int pi = i % g.nx, pj = j % g.ny, pk = (dim == 3) ? k % g.nz : 0;
    const long long P = ((long long)pk * g.ny + pj) * g.nx + pi;
    for (int q = 0; q < dim; ++q) dof[(size_t)n * dim + q] = (P == 0) ? -1 - q : (int)(dim * P - dim + q);
    return;
  }
  // Dirichlet: x on i = 0 and i = nx, every direction of node 0
  const long long before = 2LL * (n / sx) + ((n % sx) > 0 ? 1 : 0) + (n > 0 ? dim - 1 : 0);
  const long long free_before = (long long)dim * n - before;
  long long f = free_before, p = before;
  for (int q = 0; q < dim; ++q) {
    const bool c = (n == 0) || (q == 0 && (i == 0 || i == g.nx));
    if (c) dof[(size_t)n * dim + q] = (int)(-1 - p++);
    else dof[(size_t)n * dim + q] = (int)f++;
  }
}

}  // namespace pgp

namespace pg {

namespace {
struct DevBuf {
  void* p = nullptr;
  cudaStream_t st;
  explicit DevBuf(cudaStream_t s) : st(s) {}
  ~DevBuf() { if (p) cudaFreeAsync(p, st); }
};
}  // namespace

// Runs the device passes for the structured mesh of d; fills pr (pr.valid on success).  Returns
// 0, or a PG_ERR_DEVICE-style nonzero with err set when a CUDA call fails.
int device_prep(const ProblemDesc& d, PrepResult& pr, std::string& err) {
  pr = PrepResult();
  const int dim = (d.elem_type == TET4) ? 3 : 2;
  pgp::Grid g{};
  g.dim = dim;
  g.etype = d.elem_type;
  g.nx = d.n[0]; g.ny = d.n[1]; g.nz = (dim == 3) ? d.n[2] : 0;
  for (int q = 0; q < 3; ++q) { g.lo[q] = d.lo[q]; g.h[q] = (q < dim) ? (d.hi[q] - d.lo[q]) / d.n[q] : 0.0; }
  g.ninc = (int)(d.incl.size() / (dim + 1));
  // (grids of fewer than 2 cells per direction, where edge offsets coincide, stay on the host)
  if (g.nx < 2 || g.ny < 2 || (dim == 3 && g.nz < 2)) return 0;
  const long long nstd_ll = (long long)(g.nx + 1) * (g.ny + 1) * (g.nz + 1);
  if (nstd_ll > 400000000LL) { err = "mesh too large"; return 2; }
  const int n_std = (int)nstd_ll;
  const long long ne_ll = (d.elem_type == TRI3) ? 2LL * g.nx * g.ny : (d.elem_type == QUAD4 ? (long long)g.nx * g.ny : 6LL * g.nx * g.ny * g.nz);
  const int ne = (int)ne_ll;
  const int ndir = (dim == 2) ? pgp::kDirs2 : pgp::kDirs3;
  const size_t nflag = (size_t)n_std * ndir * 2;
  const size_t ntiles = (nflag + pgp::kScanTile - 1) / pgp::kScanTile;

  cudaStream_t st;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) { err = "cudaStreamCreate failed"; return 10; }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, st);
  // one allocation carved into the arrays (each 256-byte aligned)
  auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
  const size_t b_incl = al(std::max<size_t>(1, d.incl.size()) * sizeof(double));
  const size_t b_det = al((size_t)n_std * sizeof(int)), b_flag = al((size_t)ne), b_mark = al(nflag);
  const size_t b_eincl = al(nflag * sizeof(int)), b_tiles = al((ntiles + 1) * sizeof(int)), b_small = 256;
  const size_t b_list = al(nflag * sizeof(int)), b_dof = al((size_t)n_std * dim * sizeof(int));
  const size_t total = b_incl + b_det + b_flag + b_mark + b_eincl + b_tiles + b_small + b_list + b_dof;
  int rc = 0;
  {
    DevBuf buf(st);
    if (cudaMallocAsync(&buf.p, total, st) != cudaSuccess) { err = "device memory for the preprocessing"; rc = 10; }
    if (!rc) {
      char* p = static_cast<char*>(buf.p);
      double* d_incl = reinterpret_cast<double*>(p); p += b_incl;
      int* d_det = reinterpret_cast<int*>(p); p += b_det;
      unsigned char* d_flag = reinterpret_cast<unsigned char*>(p); p += b_flag;
      unsigned char* d_mark = reinterpret_cast<unsigned char*>(p); p += b_mark;
      int* d_eincl = reinterpret_cast<int*>(p); p += b_eincl;
      int* d_tiles = reinterpret_cast<int*>(p); p += b_tiles;
      int* d_small = reinterpret_cast<int*>(p); p += b_small;   // surface, rule_ok, bad_edge, n_enr, no_sign
      int* d_list = reinterpret_cast<int*>(p); p += b_list;
      int* d_dof = reinterpret_cast<int*>(p); p += b_dof;
      if (!d.incl.empty()) cudaMemcpyAsync(d_incl, d.incl.data(), d.incl.size() * sizeof(double), cudaMemcpyHostToDevice, st);
      g.incl = d_incl;
      const int init[5] = {0x7fffffff, 1, 0, 0, 0x7fffffff};
      cudaMemcpyAsync(d_small, init, sizeof(init), cudaMemcpyHostToDevice, st);
      cudaMemsetAsync(d_mark, 0, nflag, st);
      pgp::k_prep_nodes<<<(n_std + 255) / 256, 256, 0, st>>>(g, n_std, d_det, d_small + 0);
      pgp::k_prep_elems<<<(ne + 255) / 256, 256, 0, st>>>(g, ne, d_det, d_flag, d_mark, d_eincl, d_small + 1, d_small + 2);
      pgp::k_prep_dofs<<<(n_std + 255) / 256, 256, 0, st>>>(g, n_std, d.subscale, d_dof);
      pgp::k_scan_count<<<(unsigned)ntiles, pgp::kScanThreads, 0, st>>>(d_mark, nflag, d_tiles);
      pgp::k_scan_tiles<<<1, pgp::kScanThreads, 0, st>>>(d_tiles, (int)ntiles, d_small + 3);
      pgp::k_scan_write<<<(unsigned)ntiles, pgp::kScanThreads, 0, st>>>(d_mark, nflag, d_tiles, nullptr, d_list);
      int small[5];
      cudaMemcpyAsync(small, d_small, sizeof(small), cudaMemcpyDeviceToHost, st);
      pr.node_detect.resize(n_std);
      pr.elem_flag.resize(ne);
      pr.std_dof.resize((size_t)n_std * dim);
      cudaMemcpyAsync(pr.node_detect.data(), d_det, (size_t)n_std * sizeof(int), cudaMemcpyDeviceToHost, st);
      cudaMemcpyAsync(pr.elem_flag.data(), d_flag, (size_t)ne, cudaMemcpyDeviceToHost, st);
      cudaMemcpyAsync(pr.std_dof.data(), d_dof, (size_t)n_std * dim * sizeof(int), cudaMemcpyDeviceToHost, st);
      if (cudaStreamSynchronize(st) != cudaSuccess) { err = "device preprocessing failed"; rc = 10; }
      if (!rc) {
        pr.surface_node = (small[0] == 0x7fffffff) ? -1 : small[0];
        const int n_enr = small[3];
        pr.edges_valid = small[1] == 1 && small[2] == 0 && pr.surface_node < 0;
        if (pr.edges_valid && n_enr > 0) {
          void* out = nullptr;
          const size_t b_out = al((size_t)n_enr * 3 * sizeof(int)) + al((size_t)n_enr * 3 * sizeof(double));
          if (cudaMallocAsync(&out, b_out, st) != cudaSuccess) { err = "device memory for the enrichment nodes"; rc = 10; }
          else {
            int* o_edge = static_cast<int*>(out);
            int* o_incl = o_edge + 2 * (size_t)n_enr;
            double* o_x = reinterpret_cast<double*>(static_cast<char*>(out) + al((size_t)n_enr * 3 * sizeof(int)));
            pgp::k_prep_roots<<<(n_enr + 127) / 128, 128, 0, st>>>(g, n_enr, d_list, d_eincl, o_edge, o_incl, o_x, d_small + 4);
            pr.enr_edge.resize((size_t)2 * n_enr);
            pr.enr_incl.resize(n_enr);
            pr.XE.resize((size_t)3 * n_enr);
            cudaMemcpyAsync(pr.enr_edge.data(), o_edge, (size_t)2 * n_enr * sizeof(int), cudaMemcpyDeviceToHost, st);
            cudaMemcpyAsync(pr.enr_incl.data(), o_incl, (size_t)n_enr * sizeof(int), cudaMemcpyDeviceToHost, st);
            cudaMemcpyAsync(pr.XE.data(), o_x, (size_t)3 * n_enr * sizeof(double), cudaMemcpyDeviceToHost, st);
            cudaMemcpyAsync(small, d_small, sizeof(small), cudaMemcpyDeviceToHost, st);
            cudaFreeAsync(out, st);
            if (cudaStreamSynchronize(st) != cudaSuccess) { err = "device enrichment nodes failed"; rc = 10; }
            else if (small[4] != 0x7fffffff) pr.no_sign_change = small[4];
          }
        }
      }
    }
    cudaEventRecord(e1, st);
  }
  if (!rc && cudaStreamSynchronize(st) != cudaSuccess) { err = "device preprocessing failed"; rc = 10; }
  if (!rc) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    pr.device_ms = ms;
    pr.valid = true;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamDestroy(st);
  return rc;
}

}  // namespace pg

// ------------------------------------------------------------------ adjacency and CSR pattern
// device_pattern forms what build_pattern (pg_setup.cpp) forms, from the same inputs: every
// element's DOF nodes (structured connectivity, or the cut element's node list), then
//   dn_adj    (DOF node, element * 32 + local node) keys sorted: each DOF node's entries in
//             element order;
//   dn_nbr    (DOF node, DOF node) keys of every node pair of every element, sorted, duplicates
//             dropped: each DOF node's distinct neighbours in increasing order;
//   rp / ci   per DOF node the free and constrained columns of its neighbours' DOFs, its rows'
//             lengths scanned into the four blocks' row pointers, then the columns written.
#include <cub/cub.cuh>

namespace pgp {

struct PatIn {
  Grid g;
  int npe, ne, n_dn, n_free, n_const;
  const int* cut_of;
  const int* cut_node_off;
  const int* cut_nodes;
  const int* node_dn;
  const int* dn_node;
  const int* node_dof;
};

__device__ __forceinline__ int pat_nodes(const PatIn& in, int e, int* nd) {
  const int c = in.cut_of[e];
  if (c < 0) return elem_nodes(in.g, e, nd);
  const int o = in.cut_node_off[c], m = in.cut_node_off[c + 1] - o;
  for (int a = 0; a < m; ++a) nd[a] = in.cut_nodes[o + a];
  return m;
}

__global__ void k_pat_count(PatIn in, int* m_of, int* m2_of) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= in.ne) return;
  const int c = in.cut_of[e];
  const int m = (c < 0) ? in.npe : in.cut_node_off[c + 1] - in.cut_node_off[c];
  m_of[e] = m;
  m2_of[e] = m * m;
}

__global__ void k_pat_fill(PatIn in, const int* adj_off, const int* pair_off, unsigned long long* adj_key,
                           unsigned long long* pair_key) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= in.ne) return;
  int nd[32], dn[32];
  const int m = pat_nodes(in, e, nd);
  for (int a = 0; a < m; ++a) dn[a] = in.node_dn[nd[a]];
  unsigned long long* ak = adj_key + adj_off[e];
  unsigned long long* pk = pair_key + pair_off[e];
  for (int a = 0; a < m; ++a) {
    const unsigned long long hi = (unsigned long long)(unsigned)dn[a] << 32;
    ak[a] = hi | (unsigned)(e * 32 + a);
    for (int b = 0; b < m; ++b) pk[a * m + b] = hi | (unsigned)dn[b];
  }
}

// off[d] = first position of DOF node d in the sorted keys (keys of every d in [0, n_dn) present
// or not), off[n_dn] = n; low[i] = the key's low word.
__global__ void k_pat_bounds(const unsigned long long* key, int n, int n_dn, int* off, int* low) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > n) return;
  const int d = (i < n) ? (int)(key[i] >> 32) : n_dn;
  const int dp = (i > 0) ? (int)(key[i - 1] >> 32) : -1;
  for (int x = dp + 1; x <= d; ++x) off[x] = i;
  if (i < n) low[i] = (int)(unsigned)(key[i] & 0xffffffffull);
}

// Row lengths: DOF node a's rows get, per block, the count of its neighbours' free / constrained
// DOFs.  rp[b] holds lengths at [row + 1] (the scan follows).
__global__ void k_pat_rowlen(PatIn in, const int* nbr_off, const int* nbr, int* rp0, int* rp1, int* rp2, int* rp3) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= in.n_dn) return;
  const int dim = in.g.dim;
  int cf = 0, cp = 0;
  for (int k = nbr_off[a]; k < nbr_off[a + 1]; ++k) {
    const int nbn = in.dn_node[nbr[k]];
    for (int q = 0; q < dim; ++q) { if (in.node_dof[nbn * dim + q] < in.n_free) cf++; else cp++; }
  }
  const int na = in.dn_node[a];
  for (int q = 0; q < dim; ++q) {
    const int gq = in.node_dof[na * dim + q];
    if (gq < in.n_free) { rp0[gq + 1] = cf; rp1[gq + 1] = cp; }
    else { rp2[gq - in.n_free + 1] = cf; rp3[gq - in.n_free + 1] = cp; }
  }
}

__global__ void k_pat_cols(PatIn in, const int* nbr_off, const int* nbr, const int* rp0, const int* rp1,
                           const int* rp2, const int* rp3, int* ci0, int* ci1, int* ci2, int* ci3) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= in.n_dn) return;
  const int dim = in.g.dim;
  const int na = in.dn_node[a];
  for (int q = 0; q < dim; ++q) {
    const int gq = in.node_dof[na * dim + q];
    const bool rf = gq < in.n_free;
    int pf = rf ? rp0[gq] : rp2[gq - in.n_free];
    int pp = rf ? rp1[gq] : rp3[gq - in.n_free];
    int* cif = rf ? ci0 : ci2;
    int* cip = rf ? ci1 : ci3;
    for (int k = nbr_off[a]; k < nbr_off[a + 1]; ++k) {
      const int nbn = in.dn_node[nbr[k]];
      for (int q2 = 0; q2 < dim; ++q2) {
        const int g2 = in.node_dof[nbn * dim + q2];
        if (g2 < in.n_free) cif[pf++] = g2; else cip[pp++] = g2 - in.n_free;
      }
    }
  }
}

}  // namespace pgp

namespace pg {

namespace {
// Stream-ordered allocations freed together when the scope ends.
struct DevAllocs {
  cudaStream_t st;
  std::vector<void*> p;
  bool failed = false;
  explicit DevAllocs(cudaStream_t s) : st(s) {}
  template <class T>
  T* get(size_t n) {
    void* q = nullptr;
    if (cudaMallocAsync(&q, std::max<size_t>(1, n) * sizeof(T), st) != cudaSuccess) { failed = true; return nullptr; }
    p.push_back(q);
    return static_cast<T*>(q);
  }
  ~DevAllocs() { for (void* q : p) cudaFreeAsync(q, st); }
};
template <class T>
T* upload_vec(DevAllocs& A, const std::vector<T>& v) {
  T* d = A.get<T>(v.size());
  if (d && !v.empty()) cudaMemcpyAsync(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, A.st);
  return d;
}
}  // namespace

int device_pattern(Setup& s, std::string& err, double* device_ms) {
  const int dim = s.dim;
  pgp::PatIn in{};
  in.g.dim = dim;
  in.g.etype = s.etype;
  in.g.nx = s.desc.n[0]; in.g.ny = s.desc.n[1]; in.g.nz = (dim == 3) ? s.desc.n[2] : 0;
  in.npe = s.npe; in.ne = s.ne; in.n_dn = s.n_dn; in.n_free = s.n_free; in.n_const = s.n_const;
  // element sizes and their totals (64-bit on the host: a pattern beyond int32 stops here)
  long long n_adj = 0, n_pair = 0;
  {
    std::vector<int> cm(s.ncut);
    for (int c = 0; c < s.ncut; ++c) {
      cm[c] = s.cut_node_off[c + 1] - s.cut_node_off[c];
      if (cm[c] > 32) { err = "element with more than 32 nodes"; return 8; }
      n_adj += cm[c]; n_pair += (long long)cm[c] * cm[c];
    }
    n_adj += (long long)(s.ne - s.ncut) * s.npe;
    n_pair += (long long)(s.ne - s.ncut) * s.npe * s.npe;
  }
  if (n_adj > 2147483647LL || n_pair > 2147483647LL) { err = "mesh too large"; return 2; }
  cudaStream_t st;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) { err = "cudaStreamCreate failed"; return 10; }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, st);
  int rc = 0;
  {
    DevAllocs A(st);
    in.cut_of = upload_vec(A, s.cut_of);
    in.cut_node_off = upload_vec(A, s.cut_node_off);
    in.cut_nodes = upload_vec(A, s.cut_nodes);
    in.node_dn = upload_vec(A, s.node_dn);
    in.dn_node = upload_vec(A, s.dn_node);
    in.node_dof = upload_vec(A, s.node_dof);
    const int ne = s.ne, na = (int)n_adj, np = (int)n_pair, ndn = s.n_dn;
    int* m_of = A.get<int>(ne);
    int* m2_of = A.get<int>(ne);
    int* adj_off = A.get<int>(ne);
    int* pair_off = A.get<int>(ne);
    unsigned long long* ak = A.get<unsigned long long>(na);
    unsigned long long* ak2 = A.get<unsigned long long>(na);
    unsigned long long* pk = A.get<unsigned long long>(np);
    unsigned long long* pk2 = A.get<unsigned long long>(np);
    int* adj_o = A.get<int>(ndn + 1);
    int* adj_v = A.get<int>(na);
    int* nbr_o = A.get<int>(ndn + 1);
    int* n_sel = A.get<int>(1);
    int *rp[4], *ci[4];
    const int nrows[4] = {s.n_free, s.n_free, s.n_const, s.n_const};
    for (int b = 0; b < 4; ++b) rp[b] = A.get<int>(nrows[b] + 1);
    // CUB temporary storage: the largest of the scans, sorts and the unique selection
    int dn_bits = 1;
    while ((1LL << dn_bits) <= ndn) ++dn_bits;
    size_t t1 = 0, t2 = 0, t3 = 0, t4 = 0, t5 = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, t1, m_of, adj_off, ne, st);
    cub::DeviceRadixSort::SortKeys(nullptr, t2, ak, ak2, na, 0, 32 + dn_bits, st);
    cub::DeviceRadixSort::SortKeys(nullptr, t3, pk, pk2, np, 0, 32 + dn_bits, st);
    cub::DeviceSelect::Unique(nullptr, t4, pk2, pk, n_sel, np, st);
    cub::DeviceScan::InclusiveSum(nullptr, t5, rp[0] + 1, rp[0] + 1, std::max(s.n_free, s.n_const), st);
    const size_t tb = std::max(std::max(std::max(t1, t2), std::max(t3, t4)), t5);
    void* tmp = A.get<char>(tb);
    if (A.failed) { err = "device memory for the pattern"; rc = 10; }
    if (!rc) {
      pgp::k_pat_count<<<(ne + 255) / 256, 256, 0, st>>>(in, m_of, m2_of);
      size_t tbb = tb;
      cub::DeviceScan::ExclusiveSum(tmp, tbb, m_of, adj_off, ne, st);
      tbb = tb;
      cub::DeviceScan::ExclusiveSum(tmp, tbb, m2_of, pair_off, ne, st);
      pgp::k_pat_fill<<<(ne + 127) / 128, 128, 0, st>>>(in, adj_off, pair_off, ak, pk);
      tbb = tb;
      cub::DeviceRadixSort::SortKeys(tmp, tbb, ak, ak2, na, 0, 32 + dn_bits, st);
      pgp::k_pat_bounds<<<(na + 256) / 256, 256, 0, st>>>(ak2, na, ndn, adj_o, adj_v);
      tbb = tb;
      cub::DeviceRadixSort::SortKeys(tmp, tbb, pk, pk2, np, 0, 32 + dn_bits, st);
      tbb = tb;
      cub::DeviceSelect::Unique(tmp, tbb, pk2, pk, n_sel, np, st);
      int nnb = 0;
      cudaMemcpyAsync(&nnb, n_sel, sizeof(int), cudaMemcpyDeviceToHost, st);
      if (cudaStreamSynchronize(st) != cudaSuccess) { err = "device pattern failed"; rc = 10; }
      int* nbr_v = rc ? nullptr : A.get<int>(nnb);
      if (!rc && A.failed) { err = "device memory for the pattern"; rc = 10; }
      if (!rc) {
        pgp::k_pat_bounds<<<(nnb + 256) / 256, 256, 0, st>>>(pk, nnb, ndn, nbr_o, nbr_v);
        for (int b = 0; b < 4; ++b) cudaMemsetAsync(rp[b], 0, (nrows[b] + 1) * sizeof(int), st);
        pgp::k_pat_rowlen<<<(ndn + 127) / 128, 128, 0, st>>>(in, nbr_o, nbr_v, rp[0], rp[1], rp[2], rp[3]);
        for (int b = 0; b < 4; ++b)
          if (nrows[b] > 0) {
            tbb = tb;
            cub::DeviceScan::InclusiveSum(tmp, tbb, rp[b] + 1, rp[b] + 1, nrows[b], st);
          }
        int tot[4] = {0, 0, 0, 0};
        for (int b = 0; b < 4; ++b) cudaMemcpyAsync(&tot[b], rp[b] + nrows[b], sizeof(int), cudaMemcpyDeviceToHost, st);
        if (cudaStreamSynchronize(st) != cudaSuccess) { err = "device pattern failed"; rc = 10; }
        if (!rc) {
          for (int b = 0; b < 4; ++b) ci[b] = A.get<int>(tot[b]);
          if (A.failed) { err = "device memory for the pattern"; rc = 10; }
        }
        if (!rc) {
          pgp::k_pat_cols<<<(ndn + 127) / 128, 128, 0, st>>>(in, nbr_o, nbr_v, rp[0], rp[1], rp[2], rp[3], ci[0], ci[1],
                                                              ci[2], ci[3]);
          // results
          s.dn_adj_off.resize(ndn + 1);
          s.dn_adj.resize(na);
          s.dn_nbr_off.resize(ndn + 1);
          s.dn_nbr.resize(nnb);
          cudaMemcpyAsync(s.dn_adj_off.data(), adj_o, (ndn + 1) * sizeof(int), cudaMemcpyDeviceToHost, st);
          cudaMemcpyAsync(s.dn_adj.data(), adj_v, (size_t)na * sizeof(int), cudaMemcpyDeviceToHost, st);
          cudaMemcpyAsync(s.dn_nbr_off.data(), nbr_o, (ndn + 1) * sizeof(int), cudaMemcpyDeviceToHost, st);
          cudaMemcpyAsync(s.dn_nbr.data(), nbr_v, (size_t)nnb * sizeof(int), cudaMemcpyDeviceToHost, st);
          s.nrows[0] = s.n_free; s.ncols[0] = s.n_free;
          s.nrows[1] = s.n_free; s.ncols[1] = s.n_const;
          s.nrows[2] = s.n_const; s.ncols[2] = s.n_free;
          s.nrows[3] = s.n_const; s.ncols[3] = s.n_const;
          for (int b = 0; b < 4; ++b) {
            s.rp[b].resize(nrows[b] + 1);
            s.ci[b].resize(tot[b]);
            cudaMemcpyAsync(s.rp[b].data(), rp[b], (nrows[b] + 1) * sizeof(int), cudaMemcpyDeviceToHost, st);
            if (tot[b] > 0) cudaMemcpyAsync(s.ci[b].data(), ci[b], (size_t)tot[b] * sizeof(int), cudaMemcpyDeviceToHost, st);
          }
          if (cudaStreamSynchronize(st) != cudaSuccess) { err = "device pattern failed"; rc = 10; }
        }
      }
    }
    cudaEventRecord(e1, st);
  }
  if (!rc && cudaStreamSynchronize(st) != cudaSuccess) { err = "device pattern failed"; rc = 10; }
  if (!rc && device_ms) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    *device_ms = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamDestroy(st);
  return rc;
}

}  // namespace pg
