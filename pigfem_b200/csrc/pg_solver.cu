// pg_solver.cu -- device solvers and outputs on an assembled context.
//
//   pg_pcg_solve   Jacobi-preconditioned conjugate gradients on K_ff for several right-hand sides
//                  at once (the six unit-strain load cases of a homogenization, or one Newton
//                  correction).  FP64 throughout; every inner product is a fixed-order reduction
//                  (block partials over fixed row ranges, then one ordered sum), so a right-hand
//                  side's iterates do not depend on the other right-hand sides solved with it, and
//                  each right-hand side stops updating at its own convergence.  The iteration body
//                  is captured once into a CUDA graph and replayed in chunks; the host reads one
//                  flag word per chunk.
//   pg_homogenize  volume average of the stress over the volumetric quadrature points
//                  (Problem::homogenize, src/Problem.cpp:471-484, with the stress functor of
//                  include/AssemblerSmallStrainStructural.h:31-60).
#include "pg_ctx.h"

#include <cmath>
#include <cstring>

namespace {

constexpr int kThreads = 256;
constexpr int kRowGroup = 8;          // lanes per CSR row in the matrix-vector product
constexpr int kChunk = 16;            // iterations per graph replay
// scalar slots per right-hand side in PcgWork::sc
enum { S_RZ = 0, S_PQ, S_RR, S_BB, S_ALPHA, S_BETA, S_RELRES, S_NSC };

struct PcgArgs {
  const int* rp;
  const int* ci;
  const double* val;
  int n, nrhs, nb;
  double rtol;
  const double* dinv;
  double *x, *r, *z, *p, *q;   // p interleaved by right-hand side: p[i * nrhs + s]; the others [s][n]
  double* part;   // [3][nrhs][nb]
  double* sc;     // [nrhs][S_NSC]
  int* flag;      // [0, nrhs) done, [nrhs, 2 nrhs) iterations, [2 nrhs] active count
};

__device__ __forceinline__ void block_sum(double* sh, double v, double* out) {
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int w = kThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sh[0];
  __syncthreads();
}

// Rows of block b: [b * chunk, min(n, (b + 1) * chunk)).
__device__ __forceinline__ void block_rows(int n, int nb, int* r0, int* r1) {
  const int chunk = (n + nb - 1) / nb;
  *r0 = min(n, (int)blockIdx.x * chunk);
  *r1 = min(n, *r0 + chunk);
}

__global__ void __launch_bounds__(kThreads) k_pcg_diag(const int* rp, const int* ci, const double* val, int n,
                                                       double* dinv, int* bad) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double d = 0.0;
    for (int k = rp[i]; k < rp[i + 1]; ++k)
      if (ci[k] == i) d = val[k];
    if (!(d > 0.0) || !isfinite(d)) { atomicOr(bad, 1); dinv[i] = 0.0; }
    else dinv[i] = 1.0 / d;
  }
}

// (A x)[row] with kRowGroup lanes per row, lane-strided products then a fixed shuffle tree; every
// lane of the warp calls it (valid = false gives an empty row) so the shuffles stay converged.
__device__ __forceinline__ double row_dot(const PcgArgs& a, const double* x, int row, bool valid) {
  const int lane = threadIdx.x % kRowGroup;
  double v = 0.0;
  const int k0 = valid ? a.rp[row] : 0, k1 = valid ? a.rp[row + 1] : 0;
  for (int k = k0 + lane; k < k1; k += kRowGroup) v += a.val[k] * x[a.ci[k]];
#pragma unroll
  for (int o = kRowGroup / 2; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o, kRowGroup);
  return v;  // valid in lane 0 of the group
}

// r = b - A x, z = D^-1 r, p = z; partials of r.z, b.b, r.r
__global__ void __launch_bounds__(kThreads) k_pcg_start(PcgArgs a, const double* b) {
  __shared__ double sh[kThreads];
  int r0, r1;
  block_rows(a.n, a.nb, &r0, &r1);
  const int grp = threadIdx.x / kRowGroup, lane = threadIdx.x % kRowGroup, ngrp = kThreads / kRowGroup;
  for (int s = 0; s < a.nrhs; ++s) {
    const size_t o = (size_t)s * a.n;
    double rz = 0.0, bb = 0.0, rr = 0.0;
    for (int i0 = r0; i0 < r1; i0 += ngrp) {
      const int i = i0 + grp;
      const double ax = row_dot(a, a.x + o, i, i < r1);
      if (i < r1 && lane == 0) {
        const double ri = b[o + i] - ax;
        const double zi = a.dinv[i] * ri;
        a.r[o + i] = ri; a.z[o + i] = zi; a.p[(size_t)i * a.nrhs + s] = zi;
        rz += ri * zi; bb += b[o + i] * b[o + i]; rr += ri * ri;
      }
    }
    block_sum(sh, rz, &a.part[(0 * a.nrhs + s) * a.nb + blockIdx.x]);
    block_sum(sh, bb, &a.part[(1 * a.nrhs + s) * a.nb + blockIdx.x]);
    block_sum(sh, rr, &a.part[(2 * a.nrhs + s) * a.nb + blockIdx.x]);
  }
}

// one block per right-hand side: ordered sums of the partials
__global__ void __launch_bounds__(kThreads) k_pcg_start_reduce(PcgArgs a) {
  __shared__ double sh[kThreads];
  const int s = blockIdx.x;
  double v[3];
  for (int k = 0; k < 3; ++k) {
    double t = 0.0;
    for (int i = threadIdx.x; i < a.nb; i += kThreads) t += a.part[(k * a.nrhs + s) * a.nb + i];
    block_sum(sh, t, &sh[0]);  // result lands in sh[0] after the call's last sync
    v[k] = sh[0];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    double* sc = a.sc + s * S_NSC;
    sc[S_RZ] = v[0]; sc[S_BB] = v[1]; sc[S_RR] = v[2];
    const double nb = sqrt(v[1]);
    sc[S_RELRES] = nb > 0.0 ? sqrt(v[2]) / nb : 0.0;
    const int done = (nb == 0.0) || (sc[S_RELRES] <= a.rtol);
    a.flag[s] = done;
    a.flag[a.nrhs + s] = 0;
    if (done) atomicSub(&a.flag[2 * a.nrhs], 1);
  }
}

// q = A p; partials of p.q.  The right-hand sides still iterating share one pass over the matrix
// (up to kSpmvRhs at a time): each row's values and column indices are read once and multiplied
// with every right-hand side's p, whose values for one column are adjacent (p is interleaved by
// right-hand side).  Each right-hand side's sums are the ones row_dot forms (same lane-strided
// products, same shuffle tree), so its iterates do not depend on the others.
constexpr int kSpmvRhs = 8;
__global__ void __launch_bounds__(kThreads) k_pcg_spmv(PcgArgs a) {
  __shared__ double sh[kThreads];
  if (a.flag[2 * a.nrhs] == 0) return;
  int r0, r1;
  block_rows(a.n, a.nb, &r0, &r1);
  const int grp = threadIdx.x / kRowGroup, lane = threadIdx.x % kRowGroup, ngrp = kThreads / kRowGroup;
  for (int s0 = 0; s0 < a.nrhs; s0 += kSpmvRhs) {
    const int ns = min(kSpmvRhs, a.nrhs - s0);
    bool act[kSpmvRhs];
    double pq[kSpmvRhs];
#pragma unroll
    for (int j = 0; j < kSpmvRhs; ++j) { act[j] = j < ns && !a.flag[s0 + j]; pq[j] = 0.0; }
    for (int i0 = r0; i0 < r1; i0 += ngrp) {
      const int i = i0 + grp;
      const bool valid = i < r1;
      double v[kSpmvRhs];
#pragma unroll
      for (int j = 0; j < kSpmvRhs; ++j) v[j] = 0.0;
      const int k0 = valid ? a.rp[i] : 0, k1 = valid ? a.rp[i + 1] : 0;
      for (int k = k0 + lane; k < k1; k += kRowGroup) {
        const double av = a.val[k];
        const int c = a.ci[k];
#pragma unroll
        for (int j = 0; j < kSpmvRhs; ++j)
          if (act[j]) v[j] += av * a.p[(size_t)c * a.nrhs + s0 + j];
      }
#pragma unroll
      for (int j = 0; j < kSpmvRhs; ++j) {
        if (!act[j]) continue;   // uniform over the block
#pragma unroll
        for (int o = kRowGroup / 2; o > 0; o >>= 1) v[j] += __shfl_down_sync(0xffffffffu, v[j], o, kRowGroup);
        if (valid && lane == 0) {
          a.q[(size_t)(s0 + j) * a.n + i] = v[j];
          pq[j] += a.p[(size_t)i * a.nrhs + s0 + j] * v[j];
        }
      }
    }
    for (int j = 0; j < ns; ++j)
      if (act[j]) block_sum(sh, pq[j], &a.part[(0 * a.nrhs + s0 + j) * a.nb + blockIdx.x]);
  }
}

// The same product for exactly NS right-hand sides (NS = nrhs <= 8, known at compile time): a
// column's NS values of p are read as 16-byte pairs when NS is even, and every lane keeps two
// nonzeros in flight; each right-hand side's products are still added in the lane's nonzero
// order, so the sums are those of k_pcg_spmv.
template <int NS>
__device__ __forceinline__ void load_p(const double* __restrict__ p, int c, double* out) {
  if constexpr (NS % 2 == 0) {
    const double2* q = reinterpret_cast<const double2*>(p + (size_t)c * NS);
#pragma unroll
    for (int j = 0; j < NS / 2; ++j) { const double2 t = __ldg(q + j); out[2 * j] = t.x; out[2 * j + 1] = t.y; }
  } else {
#pragma unroll
    for (int j = 0; j < NS; ++j) out[j] = __ldg(p + (size_t)c * NS + j);
  }
}

template <int NS>
__global__ void __launch_bounds__(kThreads) k_pcg_spmv_n(PcgArgs a) {
  __shared__ double sh[kThreads];
  if (a.flag[2 * a.nrhs] == 0) return;
  int r0, r1;
  block_rows(a.n, a.nb, &r0, &r1);
  const int grp = threadIdx.x / kRowGroup, lane = threadIdx.x % kRowGroup, ngrp = kThreads / kRowGroup;
  bool act[NS];
  double pq[NS];
#pragma unroll
  for (int j = 0; j < NS; ++j) { act[j] = !a.flag[j]; pq[j] = 0.0; }
  for (int i0 = r0; i0 < r1; i0 += ngrp) {
    const int i = i0 + grp;
    const bool valid = i < r1;
    double v[NS];
#pragma unroll
    for (int j = 0; j < NS; ++j) v[j] = 0.0;
    const int k0 = valid ? a.rp[i] : 0, k1 = valid ? a.rp[i + 1] : 0;
    int k = k0 + lane;
    for (; k + kRowGroup < k1; k += 2 * kRowGroup) {
      const double av0 = __ldg(a.val + k), av1 = __ldg(a.val + k + kRowGroup);
      const int c0 = __ldg(a.ci + k), c1 = __ldg(a.ci + k + kRowGroup);
      double p0[NS], p1[NS];
      load_p<NS>(a.p, c0, p0);
      load_p<NS>(a.p, c1, p1);
#pragma unroll
      for (int j = 0; j < NS; ++j) v[j] += av0 * p0[j];
#pragma unroll
      for (int j = 0; j < NS; ++j) v[j] += av1 * p1[j];
    }
    if (k < k1) {
      const double av0 = __ldg(a.val + k);
      double p0[NS];
      load_p<NS>(a.p, __ldg(a.ci + k), p0);
#pragma unroll
      for (int j = 0; j < NS; ++j) v[j] += av0 * p0[j];
    }
#pragma unroll
    for (int j = 0; j < NS; ++j) {
      if (!act[j]) continue;   // uniform over the block
#pragma unroll
      for (int o = kRowGroup / 2; o > 0; o >>= 1) v[j] += __shfl_down_sync(0xffffffffu, v[j], o, kRowGroup);
      if (valid && lane == 0) {
        a.q[(size_t)j * a.n + i] = v[j];
        pq[j] += a.p[(size_t)i * NS + j] * v[j];
      }
    }
  }
#pragma unroll
  for (int j = 0; j < NS; ++j)
    if (act[j]) block_sum(sh, pq[j], &a.part[(0 * a.nrhs + j) * a.nb + blockIdx.x]);
}

__global__ void __launch_bounds__(kThreads) k_pcg_alpha(PcgArgs a) {
  __shared__ double sh[kThreads];
  if (a.flag[2 * a.nrhs] == 0) return;
  const int s = blockIdx.x;
  if (a.flag[s]) return;
  double t = 0.0;
  for (int i = threadIdx.x; i < a.nb; i += kThreads) t += a.part[(0 * a.nrhs + s) * a.nb + i];
  block_sum(sh, t, &sh[0]);
  if (threadIdx.x == 0) {
    double* sc = a.sc + s * S_NSC;
    sc[S_PQ] = sh[0];
    sc[S_ALPHA] = sc[S_RZ] / sh[0];
  }
}

// x += alpha p, r -= alpha q, z = D^-1 r; partials of r.z and r.r
__global__ void __launch_bounds__(kThreads) k_pcg_update(PcgArgs a) {
  __shared__ double sh[kThreads];
  if (a.flag[2 * a.nrhs] == 0) return;
  int r0, r1;
  block_rows(a.n, a.nb, &r0, &r1);
  for (int s = 0; s < a.nrhs; ++s) {
    if (a.flag[s]) continue;
    const size_t o = (size_t)s * a.n;
    const double al = a.sc[s * S_NSC + S_ALPHA];
    double rz = 0.0, rr = 0.0;
    for (int i = r0 + threadIdx.x; i < r1; i += kThreads) {
      a.x[o + i] += al * a.p[(size_t)i * a.nrhs + s];
      const double ri = a.r[o + i] - al * a.q[o + i];
      const double zi = a.dinv[i] * ri;
      a.r[o + i] = ri; a.z[o + i] = zi;
      rz += ri * zi; rr += ri * ri;
    }
    block_sum(sh, rz, &a.part[(1 * a.nrhs + s) * a.nb + blockIdx.x]);
    block_sum(sh, rr, &a.part[(2 * a.nrhs + s) * a.nb + blockIdx.x]);
  }
}

__global__ void __launch_bounds__(kThreads) k_pcg_beta(PcgArgs a) {
  __shared__ double sh[kThreads];
  if (a.flag[2 * a.nrhs] == 0) return;
  const int s = blockIdx.x;
  if (a.flag[s]) return;
  double v[2];
  for (int k = 0; k < 2; ++k) {
    double t = 0.0;
    for (int i = threadIdx.x; i < a.nb; i += kThreads) t += a.part[((1 + k) * a.nrhs + s) * a.nb + i];
    block_sum(sh, t, &sh[0]);
    v[k] = sh[0];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    double* sc = a.sc + s * S_NSC;
    sc[S_BETA] = v[0] / sc[S_RZ];
    sc[S_RZ] = v[0];
    sc[S_RR] = v[1];
    sc[S_RELRES] = sqrt(v[1]) / sqrt(sc[S_BB]);
    a.flag[a.nrhs + s] += 1;
    if (sc[S_RELRES] <= a.rtol || !isfinite(sc[S_RELRES])) {
      a.flag[s] = 1;
      atomicSub(&a.flag[2 * a.nrhs], 1);
    }
  }
}

// p = z + beta p for the right-hand sides still iterating
__global__ void __launch_bounds__(kThreads) k_pcg_dir(PcgArgs a) {
  if (a.flag[2 * a.nrhs] == 0) return;
  int r0, r1;
  block_rows(a.n, a.nb, &r0, &r1);
  for (int s = 0; s < a.nrhs; ++s) {
    if (a.flag[s]) continue;
    const size_t o = (size_t)s * a.n;
    const double be = a.sc[s * S_NSC + S_BETA];
    for (int i = r0 + threadIdx.x; i < r1; i += kThreads) {
      double& pi = a.p[(size_t)i * a.nrhs + s];
      pi = a.z[o + i] + be * pi;
    }
  }
}

void launch_iteration(const PcgArgs& a, cudaStream_t st) {
  switch (a.nrhs) {
    case 1: k_pcg_spmv_n<1><<<a.nb, kThreads, 0, st>>>(a); break;
    case 2: k_pcg_spmv_n<2><<<a.nb, kThreads, 0, st>>>(a); break;
    case 3: k_pcg_spmv_n<3><<<a.nb, kThreads, 0, st>>>(a); break;
    case 4: k_pcg_spmv_n<4><<<a.nb, kThreads, 0, st>>>(a); break;
    case 6: k_pcg_spmv_n<6><<<a.nb, kThreads, 0, st>>>(a); break;
    default: k_pcg_spmv<<<a.nb, kThreads, 0, st>>>(a); break;
  }
  k_pcg_alpha<<<a.nrhs, kThreads, 0, st>>>(a);
  k_pcg_update<<<a.nb, kThreads, 0, st>>>(a);
  k_pcg_beta<<<a.nrhs, kThreads, 0, st>>>(a);
  k_pcg_dir<<<a.nb, kThreads, 0, st>>>(a);
}

int pcg_reserve(pg_ctx* c, int nrhs) {
  PcgWork& w = c->pcg;
  const int n = c->s.n_free;
  if (w.cap_rhs >= nrhs && w.n == n) return 0;
  if (!w.stream) {
    if (cudaStreamCreateWithFlags(&w.stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&w.ev, cudaEventDisableTiming) != cudaSuccess)
      return pg_set_err(c, PG_ERR_DEVICE, "solver stream creation failed");
    if (cudaMallocHost(&w.hflag, sizeof(int) * 64) != cudaSuccess) return pg_set_err(c, PG_ERR_DEVICE, "pinned flag allocation failed");
  }
  w.n = n;
  w.cap_rhs = nrhs;
  w.nb = 8 * 148;   // row ranges: enough blocks in flight to hide the matrix-vector latency
  int rc = 0;
  if (!w.dinv) rc |= pg_dalloc(c, (size_t)n, &w.dinv);
  if (!w.ci) {
    // column indices of K_ff (the assembly writes values by slot and never needs them)
    int* ci = nullptr;
    rc |= pg_dalloc(c, c->s.ci[0].size(), &ci);
    if (!rc && !c->s.ci[0].empty() &&
        cudaMemcpyAsync(ci, c->s.ci[0].data(), c->s.ci[0].size() * sizeof(int), cudaMemcpyHostToDevice, c->up) != cudaSuccess)
      rc = 1;
    w.ci = ci;
  }
  rc |= pg_dalloc(c, (size_t)n * nrhs, &w.r);
  rc |= pg_dalloc(c, (size_t)n * nrhs, &w.z);
  rc |= pg_dalloc(c, (size_t)n * nrhs, &w.p);
  rc |= pg_dalloc(c, (size_t)n * nrhs, &w.q);
  rc |= pg_dalloc(c, (size_t)3 * nrhs * w.nb, &w.part);
  rc |= pg_dalloc(c, (size_t)S_NSC * nrhs, &w.sc);
  rc |= pg_dalloc(c, (size_t)2 * nrhs + 1, &w.flag);
  if (rc) return PG_ERR_DEVICE;
  return pg_alloc_sync(c);
}

// ---------------------------------------------------------------- homogenization
constexpr int kHomBlocks = 2 * 148;

// Per block: sum over a fixed element range of w * sigma (NV entries) and w.
template <int DIM>
__global__ void __launch_bounds__(kThreads) k_homogenize(pgd::DevProblem P, const double* U, double* part) {
  constexpr int NPE = DIM + 1;
  constexpr int NV = (DIM == 2) ? 3 : 6;
  __shared__ double sh[kThreads];
  const int chunk = (P.ne + gridDim.x - 1) / gridDim.x;
  const int e0 = min(P.ne, (int)blockIdx.x * chunk), e1 = min(P.ne, e0 + chunk);
  double acc[NV + 1];
#pragma unroll
  for (int v = 0; v <= NV; ++v) acc[v] = 0.0;
  for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
    const int cc = P.cut_of[e];
    if (DIM == 2 && cc < 0 && P.npe == 4) {
      // uncut quad4: the four Gauss points of its bilinear map
      double x[4][2], u[4][2];
#pragma unroll
      for (int n = 0; n < 4; ++n) {
        const int id = P.conn[(size_t)e * 4 + n];
#pragma unroll
        for (int d = 0; d < 2; ++d) { x[n][d] = P.X[(size_t)id * 2 + d]; u[n][d] = U[(size_t)id * 2 + d]; }
      }
#pragma unroll
      for (int qp = 0; qp < 4; ++qp) {
        double g[4][2], w, eps[3];
        pgd::quad4_point(x, qp, g, &w);
#pragma unroll
        for (int v = 0; v < 3; ++v) eps[v] = P.subscale ? P.eps_macro[v] : 0.0;
#pragma unroll
        for (int n = 0; n < 4; ++n) pgd::add_strain<2, double>(g[n], u[n], eps);
        double sig[3];
        pgd::lei_stress<2, double>(P.Dd + 36 * P.emat[e], eps, sig);
#pragma unroll
        for (int v = 0; v < 3; ++v) acc[v] += w * sig[v];
        acc[NV] += w;
      }
    } else if (cc < 0) {
      double x[NPE][DIM], g[NPE][DIM], J, eps[NV];
      int nd[NPE];
#pragma unroll
      for (int n = 0; n < NPE; ++n) {
        nd[n] = P.conn[(size_t)e * NPE + n];
#pragma unroll
        for (int d = 0; d < DIM; ++d) x[n][d] = P.X[(size_t)nd[n] * DIM + d];
      }
      pgd::simplex_geom<DIM, double>(x, g, &J);
      const double w = J * ((DIM == 2) ? pgd::tri4_wsum() : pgd::tet5_wsum());
#pragma unroll
      for (int v = 0; v < NV; ++v) eps[v] = P.subscale ? P.eps_macro[v] : 0.0;
#pragma unroll
      for (int n = 0; n < NPE; ++n) {
        double u[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) u[d] = U[(size_t)nd[n] * DIM + d];
        pgd::add_strain<DIM, double>(g[n], u, eps);
      }
      double sig[NV];
      pgd::lei_stress<DIM, double>(P.Dd + 36 * P.emat[e], eps, sig);
#pragma unroll
      for (int v = 0; v < NV; ++v) acc[v] += w * sig[v];
      acc[NV] += w;
    } else {
      const int mn = P.cut_node_off[cc + 1] - P.cut_node_off[cc];
      const int* cn = P.cut_nodes + P.cut_node_off[cc];
      for (int qq = P.cut_qp_off[cc]; qq < P.cut_qp_off[cc + 1]; ++qq) {
        const double* gq = P.qp_grad + P.qp_grad_off[qq];
        double eps[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) eps[v] = P.subscale ? P.eps_macro[v] : 0.0;
        for (int n = 0; n < mn; ++n) {
          double u[DIM], gn[DIM];
#pragma unroll
          for (int d = 0; d < DIM; ++d) { u[d] = U[(size_t)cn[n] * DIM + d]; gn[d] = gq[n * DIM + d]; }
          pgd::add_strain<DIM, double>(gn, u, eps);
        }
        double sig[NV];
        pgd::lei_stress<DIM, double>(P.Dd + 36 * P.qp_mat[qq], eps, sig);
        const double w = P.qp_wgt[qq];
#pragma unroll
        for (int v = 0; v < NV; ++v) acc[v] += w * sig[v];
        acc[NV] += w;
      }
    }
  }
  for (int v = 0; v <= NV; ++v) block_sum(sh, acc[v], &part[(size_t)v * gridDim.x + blockIdx.x]);
}

__global__ void k_homogenize_final(const double* part, int nb, int nv, double* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double vol = 0.0;
  for (int i = 0; i < nb; ++i) vol += part[(size_t)nv * nb + i];
  for (int v = 0; v < nv; ++v) {
    double s = 0.0;
    for (int i = 0; i < nb; ++i) s += part[(size_t)v * nb + i];
    out[v] = s / vol;
  }
  out[nv] = vol;
}

}  // namespace

extern "C" {

int pg_pcg_solve(pg_ctx* c, const double* d_b, double* d_x, int nrhs, double rtol, int max_it, int* iters,
                 double* relres) {
  if (!c || !d_b || !d_x || nrhs < 1 || nrhs > 16 || !(rtol > 0.0) || max_it < 1) return PG_ERR_INPUT;
  if (!pg_resident(c)) return pg_set_err(c, PG_ERR_STATE, "the context has no device residency (pg_upload it first)");
  if (!c->assembled) return pg_set_err(c, PG_ERR_STATE, "assemble K before solving with it");
  if (c->s.n_free == 0) return pg_set_err(c, PG_ERR_STATE, "no free degrees of freedom");
  if (int rc = pcg_reserve(c, nrhs)) return rc;
  PcgWork& w = c->pcg;
  const int n = c->s.n_free;
  // order after the assembly on the context's stream
  cudaEventRecord(w.ev, c->stream);
  cudaStreamWaitEvent(w.stream, w.ev, 0);
  PcgArgs a{c->P.rp[0], w.ci, c->P.val[0], n, nrhs, w.nb, rtol,
            w.dinv, d_x, w.r, w.z, w.p, w.q, w.part, w.sc, w.flag};
  // the diagonal changes with every assembly: recompute it
  cudaMemsetAsync(w.flag, 0, sizeof(int) * (2 * nrhs + 1), w.stream);
  k_pcg_diag<<<2 * 148, kThreads, 0, w.stream>>>(a.rp, a.ci, a.val, n, w.dinv, w.flag + 2 * nrhs);
  cudaMemcpyAsync(w.hflag, w.flag + 2 * nrhs, sizeof(int), cudaMemcpyDeviceToHost, w.stream);
  if (cudaStreamSynchronize(w.stream) != cudaSuccess) return pg_set_err(c, PG_ERR_DEVICE, "solver set-up failed");
  if (w.hflag[0]) return pg_set_err(c, PG_ERR_NONFINITE, "K_ff has a non-positive or non-finite diagonal entry");
  const int active = nrhs;
  cudaMemcpyAsync(w.flag + 2 * nrhs, &active, sizeof(int), cudaMemcpyHostToDevice, w.stream);
  k_pcg_start<<<w.nb, kThreads, 0, w.stream>>>(a, d_b);
  k_pcg_start_reduce<<<nrhs, kThreads, 0, w.stream>>>(a);
  // capture kChunk iterations once, replay until every right-hand side is done or max_it
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  if (cudaStreamBeginCapture(w.stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
    return pg_set_err(c, PG_ERR_DEVICE, "graph capture failed to start");
  for (int it = 0; it < kChunk; ++it) launch_iteration(a, w.stream);
  if (cudaStreamEndCapture(w.stream, &graph) != cudaSuccess || cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    return pg_set_err(c, PG_ERR_DEVICE, "graph instantiation failed");
  }
  int done_iters = 0;
  int rc = 0;
  while (true) {
    cudaMemcpyAsync(w.hflag, w.flag + 2 * nrhs, sizeof(int), cudaMemcpyDeviceToHost, w.stream);
    if (cudaStreamSynchronize(w.stream) != cudaSuccess) { rc = pg_set_err(c, PG_ERR_DEVICE, "solver iteration failed"); break; }
    if (w.hflag[0] == 0 || done_iters >= max_it) break;
    cudaGraphLaunch(exec, w.stream);
    done_iters += kChunk;
  }
  cudaGraphExecDestroy(exec);
  cudaGraphDestroy(graph);
  if (rc) return rc;
  // results
  std::vector<int> fl(2 * nrhs + 1);
  std::vector<double> sc((size_t)S_NSC * nrhs);
  cudaMemcpyAsync(fl.data(), w.flag, sizeof(int) * fl.size(), cudaMemcpyDeviceToHost, w.stream);
  cudaMemcpyAsync(sc.data(), w.sc, sizeof(double) * sc.size(), cudaMemcpyDeviceToHost, w.stream);
  if (cudaStreamSynchronize(w.stream) != cudaSuccess) return pg_set_err(c, PG_ERR_DEVICE, "solver read-back failed");
  // later work on the context's stream sees the solution
  cudaEventRecord(w.ev, w.stream);
  cudaStreamWaitEvent(c->stream, w.ev, 0);
  bool all = true;
  for (int s = 0; s < nrhs; ++s) {
    if (iters) iters[s] = fl[nrhs + s];
    if (relres) relres[s] = sc[(size_t)s * S_NSC + S_RELRES];
    all = all && fl[s] && std::isfinite(sc[(size_t)s * S_NSC + S_RELRES]);
  }
  if (!all) return pg_set_err(c, PG_ERR_STATE, "PCG did not reach the tolerance within max_it");
  return 0;
}

int pg_homogenize(pg_ctx* c, const double* d_U, double t_frac, double* out) {
  if (!c || !d_U || !out) return PG_ERR_INPUT;
  if (!pg_resident(c)) return pg_set_err(c, PG_ERR_STATE, "the context has no device residency (pg_upload it first)");
  const int dim = c->s.dim, nv = dim == 2 ? 3 : 6;
  if (!c->d_hom && (pg_dalloc(c, (size_t)(nv + 2) * kHomBlocks + 8, &c->d_hom) || pg_alloc_sync(c))) return PG_ERR_DEVICE;
  pgd::DevProblem P = c->P;
  for (int v = 0; v < 6; ++v) P.eps_macro[v] = c->s.desc.eps_macro[v] * t_frac;
  if (dim == 2) k_homogenize<2><<<kHomBlocks, kThreads, 0, c->stream>>>(P, d_U, c->d_hom);
  else k_homogenize<3><<<kHomBlocks, kThreads, 0, c->stream>>>(P, d_U, c->d_hom);
  double* res = c->d_hom + (size_t)(nv + 1) * kHomBlocks;
  k_homogenize_final<<<1, 32, 0, c->stream>>>(c->d_hom, kHomBlocks, nv, res);
  double h[7];
  cudaMemcpyAsync(h, res, sizeof(double) * (nv + 1), cudaMemcpyDeviceToHost, c->stream);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return pg_set_err(c, PG_ERR_DEVICE, "homogenization failed");
  std::memcpy(out, h, sizeof(double) * (nv + 1));
  return 0;
}

}  // extern "C"
