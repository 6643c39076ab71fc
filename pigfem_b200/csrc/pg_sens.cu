// pg_sens.cu -- material sensitivity of the internal force: the reference's second element loop
// (SensitivityParameter::assemble_dPdd, src/SensitivityParameter.cpp:110-153, with
// SensitivityMaterialParameter::assemble_elem_dPdd, src/SensitivityMaterialParameter.cpp:41-220,
// and SensitivityMaterialParameterStructural::KernelVolumetric,
// src/SensitivityMaterialParameterStructural.cpp:17-37) for a parameter p of a linear elastic
// isotropic bulk material m:
//
//   dP/dp = sum over the points of the elements and sub-elements of material m of
//           w B^T (dD/dp eps),  eps = B u.
//
// Three launches on the context's stream, no atomics:
//   k_sens_uncut  a thread per uncut element of material m: its NPE x DIM values;
//   k_sens_cut    a thread per (cut element, element node): the sum over the element's listed
//                 points (the host lists, per call, the points of the sub-elements of material m
//                 with their weights and the point whose gradients the reference reads there);
//   k_sens_rows   a thread per DOF node: the values of its (element, local node) adjacency
//                 entries summed in adjacency order into dP_f / dP_p.
// The cut elements follow the reference as written: for the q-th point of a sub-element the
// gradients are those of the element's q-th point while the weight is the point's own
// (src/SensitivityMaterialParameter.cpp:131-141 index the shape gradients by the sub-element's
// point index and J, W by the running index).
#include "pg_ctx.h"
#include "pg_kernels.cuh"

#include <algorithm>
#include <vector>

namespace pgd {

template <int DIM>
__device__ __forceinline__ void sens_stress(const double* __restrict__ Q, const double* eps, double* ds) {
  constexpr int NV = (DIM == 2) ? 3 : 6;
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    double a = 0.0;
#pragma unroll
    for (int j = 0; j < NV; ++j) a += __ldg(&Q[i * NV + j]) * eps[j];
    ds[i] = a;
  }
}

template <int DIM, int NPE>
__global__ void __launch_bounds__(128) k_sens_uncut(DevProblem P, const double* __restrict__ U, int m,
                                                    const double* __restrict__ Q, double* __restrict__ out) {
  constexpr int NV = (DIM == 2) ? 3 : 6;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= P.ne || __ldg(&P.cut_of[e]) >= 0 || __ldg(&P.emat[e]) != m) return;
  double x[NPE][DIM], u[NPE][DIM], r[NPE][DIM];
#pragma unroll
  for (int n = 0; n < NPE; ++n) {
    const int id = __ldg(&P.conn[(size_t)e * NPE + n]);
    load_node<DIM>(P.X, id, x[n]);
    load_node<DIM>(U, id, u[n]);
#pragma unroll
    for (int d = 0; d < DIM; ++d) r[n][d] = 0.0;
  }
  if constexpr (NPE == DIM + 1) {
    // affine element: one gradient set, the rule's weights summed
    double g[NPE][DIM], J;
    simplex_geom<DIM, double>(x, g, &J);
    const double w = J * ((DIM == 2) ? tri4_wsum() : tet5_wsum());
    double eps[NV], ds[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) eps[v] = 0.0;
#pragma unroll
    for (int n = 0; n < NPE; ++n) add_strain<DIM, double>(g[n], u[n], eps);
    sens_stress<DIM>(Q, eps, ds);
#pragma unroll
    for (int n = 0; n < NPE; ++n)
#pragma unroll
      for (int q = 0; q < DIM; ++q) r[n][q] = w * bt_sig<DIM, double>(g[n], ds, q);
  } else {
    // quad4: the 2 x 2 Gauss points, each with its own gradients
#pragma unroll
    for (int qp = 0; qp < 4; ++qp) {
      double g[4][2], w;
      quad4_point(reinterpret_cast<const double(*)[2]>(x), qp, g, &w);
      double eps[3] = {0.0, 0.0, 0.0}, ds[3];
#pragma unroll
      for (int n = 0; n < 4; ++n) add_strain<2, double>(g[n], u[n], eps);
      sens_stress<2>(Q, eps, ds);
#pragma unroll
      for (int n = 0; n < 4; ++n)
#pragma unroll
        for (int q = 0; q < 2; ++q) r[n][q] += w * bt_sig<2, double>(g[n], ds, q);
    }
  }
  double* o = out + (size_t)e * NPE * DIM;
#pragma unroll
  for (int n = 0; n < NPE; ++n)
#pragma unroll
    for (int q = 0; q < DIM; ++q) o[n * DIM + q] = r[n][q];
}

template <int DIM>
__global__ void __launch_bounds__(128) k_sens_cut(DevProblem P, const double* __restrict__ U, const double* __restrict__ Q,
                                                  const int* __restrict__ pt_off, const double* __restrict__ pt_w,
                                                  const int* __restrict__ pt_g, const int* __restrict__ g_off,
                                                  const double* __restrict__ g, double* __restrict__ out) {
  constexpr int NV = (DIM == 2) ? 3 : 6;
  const int n_slots = __ldg(&P.cut_node_off[P.ncut]);
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_slots) return;
  // the cut element holding node slot t
  int lo = 0, hi = P.ncut - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (__ldg(&P.cut_node_off[mid]) <= t) lo = mid; else hi = mid - 1;
  }
  const int c = lo, n0 = __ldg(&P.cut_node_off[c]), mn = __ldg(&P.cut_node_off[c + 1]) - n0, la = t - n0;
  double r[DIM];
#pragma unroll
  for (int q = 0; q < DIM; ++q) r[q] = 0.0;
  for (int k = __ldg(&pt_off[c]); k < __ldg(&pt_off[c + 1]); ++k) {
    const double* gp = g + __ldg(&g_off[__ldg(&pt_g[k])]);
    double eps[NV], ds[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) eps[v] = 0.0;
    for (int b = 0; b < mn; ++b) {
      double gb[DIM], ub[DIM];
#pragma unroll
      for (int d = 0; d < DIM; ++d) gb[d] = __ldg(&gp[b * DIM + d]);
      load_node<DIM>(U, __ldg(&P.cut_nodes[n0 + b]), ub);
      add_strain<DIM, double>(gb, ub, eps);
    }
    sens_stress<DIM>(Q, eps, ds);
    double ga[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) ga[d] = __ldg(&gp[la * DIM + d]);
    const double w = __ldg(&pt_w[k]);
#pragma unroll
    for (int q = 0; q < DIM; ++q) r[q] += w * bt_sig<DIM, double>(ga, ds, q);
  }
#pragma unroll
  for (int q = 0; q < DIM; ++q) out[(size_t)t * DIM + q] = r[q];
}

template <int DIM, int NPE>
__global__ void __launch_bounds__(128) k_sens_rows(DevProblem P, int m, const double* __restrict__ uncut,
                                                   const double* __restrict__ cut, double* __restrict__ dPf,
                                                   double* __restrict__ dPp) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= P.n_dn) return;
  double r[DIM];
#pragma unroll
  for (int q = 0; q < DIM; ++q) r[q] = 0.0;
  for (int j = __ldg(&P.dn_adj_off[a]); j < __ldg(&P.dn_adj_off[a + 1]); ++j) {
    const int ent = __ldg(&P.dn_adj[j]);
    const int e = ent >> 5, la = ent & 31;
    const int c = __ldg(&P.cut_of[e]);
    const double* v;
    if (c >= 0) v = cut + ((size_t)__ldg(&P.cut_node_off[c]) + la) * DIM;
    else if (__ldg(&P.emat[e]) == m) v = uncut + (size_t)e * NPE * DIM + (size_t)la * DIM;
    else continue;
#pragma unroll
    for (int q = 0; q < DIM; ++q) r[q] += v[q];
  }
  const int node = __ldg(&P.dn_node[a]);
#pragma unroll
  for (int q = 0; q < DIM; ++q) {
    const int dof = __ldg(&P.node_dof[(size_t)node * DIM + q]);
    if (dof < P.n_free) dPf[dof] = r[q];
    else dPp[dof - P.n_free] = r[q];
  }
}

}  // namespace pgd

namespace {

// Device tables of the sensitivity pass, made on the first call: the per-element and per-cut-node
// values, the derivative matrices, the cut elements' unmerged point gradients, and room for a
// call's point lists.
int sens_tables(pg_ctx* c) {
  if (c->sens.ready) return 0;
  const pg::Setup& s = c->s;
  const int dim = s.dim;
  if (int rc = pg_dalloc(c, (size_t)s.ne * s.npe * dim, &c->sens.uncut)) return rc;
  if (int rc = pg_dalloc(c, (size_t)std::max(1, s.ncut ? s.cut_node_off[s.ncut] : 0) * dim, &c->sens.cut)) return rc;
  std::vector<double> dD(2 * 5 * 36);
  for (int m = 0; m < 2; ++m)
    for (int p = 0; p < 5; ++p)
      for (int i = 0; i < 36; ++i) dD[(m * 5 + p) * 36 + i] = s.dD[m][p][i];
  double* d = nullptr;
  if (int rc = pg_dalloc(c, dD.size(), &d)) return rc;
  c->sens.dD = d;
  const size_t nq = s.qp_wgt.size();
  if (int rc = pg_dalloc(c, std::max<size_t>(1, s.qp_grad.size()), &c->sens.g)) return rc;
  if (int rc = pg_dalloc(c, nq + 1, &c->sens.g_off)) return rc;
  if (int rc = pg_dalloc(c, (size_t)s.ncut + 1, &c->sens.pt_off)) return rc;
  if (int rc = pg_dalloc(c, std::max<size_t>(1, nq), &c->sens.pt_w)) return rc;
  if (int rc = pg_dalloc(c, std::max<size_t>(1, nq), &c->sens.pt_g)) return rc;
  if (int rc = pg_alloc_sync(c)) return rc;
  cudaMemcpy(c->sens.dD, dD.data(), dD.size() * sizeof(double), cudaMemcpyHostToDevice);
  if (!s.qp_grad.empty()) cudaMemcpy(c->sens.g, s.qp_grad.data(), s.qp_grad.size() * sizeof(double), cudaMemcpyHostToDevice);
  cudaMemcpy(c->sens.g_off, s.qp_grad_off.data(), s.qp_grad_off.size() * sizeof(int), cudaMemcpyHostToDevice);
  if (cudaGetLastError() != cudaSuccess) return pg_set_err(c, PG_ERR_DEVICE, "sensitivity tables: copy failed");
  c->sens.ready = true;
  return 0;
}

}  // namespace

extern "C" int pg_material_sensitivity(pg_ctx* c, const double* d_U, int material, int param, double* d_dPf,
                                       double* d_dPp) {
  if (!c || !d_U || !d_dPf || (!d_dPp && c->s.n_const)) return PG_ERR_INPUT;
  if (!pg_resident(c)) return pg_set_err(c, PG_ERR_STATE, "the context has no device residency (pg_upload it first)");
  if (material < 0 || material > 1 || param < 0 || param > 4)
    return pg_set_err(c, PG_ERR_INPUT, "material must be 0 (matrix) or 1 (fiber), param 0..4 (E, lambda, mu, K, nu)");
  if (c->s.cohesive)
    return pg_set_err(c, PG_ERR_UNSUPPORTED, "material sensitivities of cohesive problems (the laws' sensitivity "
                                             "constitutive updates) are not built");
  if (int rc = sens_tables(c)) return rc;
  const pg::Setup& s = c->s;
  // this call's point lists: the points of the sub-elements of the material, with their own
  // weights and the gradients of the element's point at the same position in the sub-element
  std::vector<int> pt_off(1, 0), pt_g;
  std::vector<double> pt_w;
  for (int cc = 0; cc < s.ncut; ++cc) {
    for (int sb = s.cut_sub_off[cc]; sb < s.cut_sub_off[cc + 1]; ++sb) {
      if (s.sub_mat[sb] != material) continue;
      for (int q = s.sub_qp_off[sb]; q < s.sub_qp_off[sb + 1]; ++q) {
        pt_w.push_back(s.qp_wgt[q]);
        pt_g.push_back(s.cut_qp_off[cc] + (q - s.sub_qp_off[sb]));
      }
    }
    pt_off.push_back((int)pt_w.size());
  }
  cudaStream_t st = c->stream;
  cudaMemcpyAsync(c->sens.pt_off, pt_off.data(), pt_off.size() * sizeof(int), cudaMemcpyHostToDevice, st);
  if (!pt_w.empty()) {
    cudaMemcpyAsync(c->sens.pt_w, pt_w.data(), pt_w.size() * sizeof(double), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(c->sens.pt_g, pt_g.data(), pt_g.size() * sizeof(int), cudaMemcpyHostToDevice, st);
  }
  const double* Q = c->sens.dD + (size_t)(material * 5 + param) * 36;
  const pgd::DevProblem& P = c->P;
  const int tpb = 128;
  const int n_slots = s.ncut ? s.cut_node_off[s.ncut] : 0;
  auto blocks = [&](long long n) { return (int)((n + tpb - 1) / tpb); };
  if (s.dim == 2 && s.npe == 3) {
    pgd::k_sens_uncut<2, 3><<<blocks(s.ne), tpb, 0, st>>>(P, d_U, material, Q, c->sens.uncut);
    if (n_slots) pgd::k_sens_cut<2><<<blocks(n_slots), tpb, 0, st>>>(P, d_U, Q, c->sens.pt_off, c->sens.pt_w, c->sens.pt_g, c->sens.g_off, c->sens.g, c->sens.cut);
    pgd::k_sens_rows<2, 3><<<blocks(s.n_dn), tpb, 0, st>>>(P, material, c->sens.uncut, c->sens.cut, d_dPf, d_dPp);
  } else if (s.dim == 2) {
    pgd::k_sens_uncut<2, 4><<<blocks(s.ne), tpb, 0, st>>>(P, d_U, material, Q, c->sens.uncut);
    if (n_slots) pgd::k_sens_cut<2><<<blocks(n_slots), tpb, 0, st>>>(P, d_U, Q, c->sens.pt_off, c->sens.pt_w, c->sens.pt_g, c->sens.g_off, c->sens.g, c->sens.cut);
    pgd::k_sens_rows<2, 4><<<blocks(s.n_dn), tpb, 0, st>>>(P, material, c->sens.uncut, c->sens.cut, d_dPf, d_dPp);
  } else {
    pgd::k_sens_uncut<3, 4><<<blocks(s.ne), tpb, 0, st>>>(P, d_U, material, Q, c->sens.uncut);
    if (n_slots) pgd::k_sens_cut<3><<<blocks(n_slots), tpb, 0, st>>>(P, d_U, Q, c->sens.pt_off, c->sens.pt_w, c->sens.pt_g, c->sens.g_off, c->sens.g, c->sens.cut);
    pgd::k_sens_rows<3, 4><<<blocks(s.n_dn), tpb, 0, st>>>(P, material, c->sens.uncut, c->sens.cut, d_dPf, d_dPp);
  }
  // the point lists are pageable host memory: wait for their copies (and the launches) here
  if (cudaStreamSynchronize(st) != cudaSuccess) return pg_set_err(c, PG_ERR_DEVICE, "sensitivity kernels failed");
  return 0;
}
