// pg_device.cuh -- device-side data layout and element physics of the B200 assembly path.
//
// Physics restated from the reference (paths relative to the PIGFEM source tree):
//   small-strain kernel ........ src/AssemblerSmallStrainStructural.cpp:23-50 (eps = B U [+ eps_macro],
//                                K = B^T D B, P = B^T sigma), B in Voigt order xx, yy, (zz), (yz, xz,) xy
//                                with engineering shear (src/Utilities.cpp:68-127)
//   linear elastic stress ...... src/material_lei.cpp:232-299 (sigma = D eps)
//   cohesive kernel ............ src/AssemblerSmallStrainStructural.cpp:86-104, src/Utilities.cpp:528-594
//   cohesive laws .............. src/Material_BilinearCohesive{,NU}.cpp, src/Material_XNCohesive{,NU}.cpp,
//                                src/Material_OPCohesive{,NU,Aug,NUAug}.cpp
//   damage zones ............... src/Material_BilinearCohesiveNU.cpp:255-266, src/Material_OPCohesiveNU.cpp:217-234,
//                                src/Material_XNCohesiveNU.cpp:264-287
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace pgd {

constexpr int kMaxNodesCut = 32;  // element-local node slots (parent + enrichment); matches the set-up encoding

enum { COH_NONE = 0, COH_BL = 1, COH_BLNU = 2, COH_XN = 3, COH_XNNU = 4, COH_OP = 5, COH_OPNU = 6, COH_OPAUG = 7, COH_OPNUAUG = 8,
       COH_TL = 9, COH_TLNU = 10, COH_STL = 11, COH_STLNU = 12 };
enum { FLAG_FUNC = 1, FLAG_JAC = 2, FLAG_FP32 = 4 };
enum { ERR_NONFINITE = 1, ERR_CUT_OVERFLOW = 2, ERR_BAD_SLOT = 4 };

struct CohConst {
  int law, nvar;
  double sigma_c, delta_c1, delta_c2, delta_cn, delta_ct, q, delta_c, beta2, alpha;
  double delta_c3;
};

// Everything one assembly launch reads or writes, as device pointers.
struct DevProblem {
  int dim, npe, nvoigt;
  int n_nodes, ne, ncut, n_dn;
  int n_free, n_const;
  int subscale;
  double D[3][36];    // bulk materials: 0 matrix, 1 fiber, 2 bounding plies
  float Df[3][36];
  const double* Dd;   // D of the three bulk materials in device memory (3 x 36), read through the L1
  const float* Dfd;
  // 2D structured tiles (pg_tile.cuh): every uncut element of the uniform grid is one of four
  // shapes (2 x cell parity + element in the cell); per shape the gradients of its three nodes, its
  // weight J W, and its element matrix per bulk material ([(la * 2 + q) * 6 + lb * 2 + q2], FP64
  // and the FP32-mixed products), formed once at upload by the element code itself
  double tile_g[4][3][2];
  double tile_w[4];
  double tile_ke[4][3][36];
  float tile_kef[4][3][36];
  CohConst coh;
  // geometry / state
  const double* X;    // n_nodes * dim
  const float* Xf;    // n_nodes * dim (FP32 copy for the mixed path)
  const double* U;    // n_nodes * dim, node-major (the reference's NodalData layout)
  const int* conn;    // ne * npe
  const int* emat;    // ne
  const int* cut_of;  // ne
  const int* node_dof;  // n_nodes * dim
  const int* node_dn;   // n_nodes
  // cut elements
  const int* cut_node_off; const int* cut_nodes;
  const int* cut_qp_off; const double* qp_wgt; const int* qp_mat; const int* qp_grad_off; const double* qp_grad;
  const int* cut_coh_off; const int* coh_nh; const int* coh_local_off; const int* coh_local;
  const int* coh_qp_off; const double* cqp_N; const double* cqp_R; const double* cqp_wgt; const int* cqp_isv;
  const int* cqp_noff;  // first shape value of each cohesive point in cqp_N (CohTri3 3, CohQuad4 4, CohEdge2 2)
  const long long* ke_off;  // per cut element: offset of its element matrix in ke
  const int* re_off;        // per cut element: offset of its first node's rows (nodes x dim)
  double* ke;               // set-up only: volumetric element matrices of the cut elements
  const double* gmac;       // set-up only: macroscale-strain response of the cut elements
  // Static part of the general rows next to cut elements (the first n_stat general nodes): the
  // cut elements' volumetric blocks summed per neighbour slot, in the slab layout [slot][q][d]
  // (stat, from stat_slot_off[node] slots on), the node id of each slot (stat_node) and the
  // summed macroscale-strain response (stat_g, dim x nvoigt per node).  The bulk laws are linear
  // elastic, so these do not depend on the state; k_general_static forms them once at set-up.
  int n_stat;
  const int* stat_slot_off;
  const int* stat_node;
  const double* stat;
  const double* stat_g;
  const double* isv_committed;
  double* isv_trial;
  uint8_t* zone;            // per cohesive qp: damage zone (0 compression, 1 loading, 2 softening, 3 failed)
  // row ownership
  const int* dn_node; const int* dn_nbr_off; const uint8_t* dn_nbr_mask;  // free-DOF bits of each neighbour
  const int* dn_adj_off; const int* dn_adj;      // adjacent (element << 5 | local node)
  const int* adj_slot32;                         // uncut elements: neighbour slot of each element node, 8 bits each
  const int* adj_slot_off; const uint8_t* adj_slots;  // all elements: neighbour slot of each element node
  const int* fast_dn; int n_fast_dn;             // DOF nodes whose elements are all uncut
  const int* tile_elem_off; const int* tile_elems; int tile_max_elems;  // elements each tile of fast nodes touches
  const uint16_t* adj_local;                     // tile-local index of each adjacency entry's element
  const int* slow_dn; int n_slow_dn;             // the remaining DOF nodes
  // Block-parallel general rows (pg_general.cuh; tri3 / tet4 meshes): one block per (general
  // node, neighbour slot), node-major: {node, slot, static index, -}; its cohesive contributions
  // [gblk_cl[b], gblk_cl[b + 1]) as (kcoh offset << 1 | negative) in adjacency order; per general
  // node the residual's traction list (kcoh offset << 1 | negative), in adjacency order.
  int n_gblk;
  const int4* gblk; const int* gblk_cl; const int* gcl;
  const int* gnode_tl_off; const int* gnode_tl;
  int maxnb_general;                             // slab slots per node in k_rows_general
  const int4* gdesc; const int* growd; const int4* adesc; const int4* aresd;  // k_rows_general descriptors
  // cohesive points
  int n_coh_qp;
  int n_coh_el;                                  // cohesive elements
  const int* ce_cut;                             // cut element of each cohesive element
  const int* coh_gnode;                          // node id of every cohesive element's local node ('-' then '+', at coh_local_off)
  const int* kc_off;                             // per cohesive element: offset of its blocks in kcoh
  double* kcoh;                                  // per call: cohesive blocks B_ab and tractions t_a
  const int* cohpos;                             // per cut-element local node: (cohesive element << 5 | position) or -1
  const int* nbr_pre;                            // per neighbour slot: free DOFs of the earlier neighbours
  int max_mn;                                    // most nodes of a cut element
  // outputs: CSR values of the four blocks and the two residual parts
  const int* rp[4];
  double* val[4];
  double* Pf; double* Pp;
  // per-call
  double eps_macro[6];
  int flags;
  int* err;
  // residual passes over several macroscale strains (pg_residual_strains): case k's strain and
  // its residual parts, [k][n_free] and [k][n_const]
  int n_cases;
  double eps_cases[6][6];
  double* Pf_cases;
  double* Pp_cases;
};

// ---------------------------------------------------------------- cohesive laws (FP64)
// x^2 as one correctly rounded product (what pow(x, 2) returns on the reference's host).
__device__ __forceinline__ double sq(double x) { return x * x; }

// Effective traction of the trilinear laws at effective opening d: linear rise to sigma_c at
// delta_c1, plateau to delta_c2, linear fall to 0 at delta_c3
// (src/Material_TrilinearCohesiveNU.cpp:90-113); the smoothed laws rise along 2v - v^2 and fall
// along 2v^3 - 3v^2 + 1 (src/Material_SmoothedTrilinearCohesiveNU.cpp:98-121).  `unload` gives
// the traction at a historical maximum as the unloading branches write it
// (src/Material_TrilinearCohesive.cpp:90-98, src/Material_SmoothedTrilinearCohesive.cpp:97-113).
__device__ inline void trilinear_curve(const CohConst& c, bool smooth, bool unload, double d, double* t, double* dt) {
  *dt = 0.0;
  if (d >= 0 && d < c.delta_c1) {
    if (smooth) {
      const double v = d / c.delta_c1;
      *t = c.sigma_c * (2.0 * v - sq(v));
      *dt = c.sigma_c * ((2.0 / c.delta_c1) * (1.0 - v));
    } else {
      *t = unload ? d * (c.sigma_c / c.delta_c1) : c.sigma_c * (d / c.delta_c1);
      *dt = c.sigma_c / c.delta_c1;
    }
  } else if (d >= c.delta_c1 && d < c.delta_c2) {
    *t = c.sigma_c;
  } else if (d >= c.delta_c2 && d < c.delta_c3) {
    if (smooth) {
      const double v = (d - c.delta_c2) / (c.delta_c3 - c.delta_c2);
      *t = c.sigma_c * (2.0 * pow(v, 3.0) - 3.0 * sq(v) + 1.0);
      *dt = c.sigma_c * (6.0 * (v / (c.delta_c3 - c.delta_c2)) * (v - 1.0));
    } else {
      *t = c.sigma_c * (1 - (d - c.delta_c2) / (c.delta_c3 - c.delta_c2));
      *dt = -1.0 * (c.sigma_c / (c.delta_c3 - c.delta_c2));
    }
  } else {
    *t = 0.0;
  }
}
// delta (dim entries, tangential first, normal last) may be overwritten by the 1e-20 clamp, as the
// reference's getDeltaEff / getDnDt do.  T gets the traction, Dm the dim x dim tangent (row-major),
// isv the trial internal variables of this quadrature point (updated in place), zone the damage zone.
__device__ inline void coh_law(const CohConst& c, int dim, double* delta, double* T, double* Dm, double* isv, uint8_t* zone) {
  double nrm = 0.0;
  for (int i = 0; i < dim; ++i) nrm += delta[i] * delta[i];
  if (nrm < 1e-40)
    for (int i = 0; i < dim; ++i) delta[i] = 1e-20;
  const int law = c.law;
  if (law == COH_XN || law == COH_XNNU) {
    const double Dn = delta[dim - 1];
    const double Dt = (dim == 2) ? delta[0] : sqrt(sq(delta[0]) + sq(delta[1]));
    const double phi_n = c.sigma_c * c.delta_cn * exp(1.0);
    double Tn, dTndDn, Tt, dTtdDt;
    const double dTndDt = 0.0, dTtdDn = 0.0;
    if (law == COH_XNNU) {
      const double shear_rat = Dt / c.delta_ct;
      const double shear_rat_exp = exp(-sq(shear_rat));
      const double norm_rat = Dn / c.delta_cn;
      const double norm_rat_exp = exp(-1.0 * norm_rat);
      Tn = (phi_n / c.delta_cn) * norm_rat_exp * norm_rat;
      Tt = (2.0 * phi_n * Dt / sq(c.delta_ct)) * c.q * shear_rat_exp;
      dTndDn = (phi_n / c.delta_cn) * norm_rat_exp * ((1 - norm_rat) / c.delta_cn);
      dTtdDt = (2.0 * phi_n / sq(c.delta_ct)) * c.q * (1 - 2.0 * sq(shear_rat)) * shear_rat_exp;
    } else {
      double& Dn_max = isv[0];
      double& Dt_max = isv[1];
      if (Dn >= Dn_max || Dn <= 0) {
        const double norm_rat = Dn / c.delta_cn;
        const double norm_rat_exp = exp(-1.0 * norm_rat);
        Tn = (phi_n / c.delta_cn) * norm_rat_exp * norm_rat;
        dTndDn = (phi_n / c.delta_cn) * norm_rat_exp * ((1 - norm_rat) / c.delta_cn);
        Dn_max = Dn;
      } else {
        const double norm_rat_max = Dn_max / c.delta_cn;
        const double norm_rat_exp_max = exp(-1.0 * norm_rat_max);
        const double Tn_max = (phi_n / c.delta_cn) * norm_rat_exp_max * norm_rat_max;
        Tn = (Dn / Dn_max) * Tn_max;
        dTndDn = Tn_max / Dn_max;
      }
      if (fabs(Dt) >= Dt_max) {
        const double shear_rat = Dt / c.delta_ct;
        const double shear_rat_exp = exp(-sq(shear_rat));
        Tt = (2.0 * phi_n * c.q / c.delta_ct) * shear_rat_exp * shear_rat;
        dTtdDt = (2.0 * phi_n / sq(c.delta_ct)) * c.q * (1 - 2.0 * sq(shear_rat)) * shear_rat_exp;
        Dt_max = fabs(Dt);
      } else {
        const double shear_rat_max = Dt_max / c.delta_ct;
        const double shear_rat_exp_max = exp(-sq(shear_rat_max));
        const double Tt_max = (2.0 * phi_n * c.q / c.delta_ct) * shear_rat_exp_max * shear_rat_max;
        Tt = (Dt / Dt_max) * Tt_max;
        dTtdDt = Tt_max / Dt_max;
      }
    }
    T[dim - 1] = Tn;
    if (dim == 2) {
      T[0] = Tt;
      Dm[0] = dTtdDt; Dm[1] = dTtdDn; Dm[2] = dTndDt; Dm[3] = dTndDn;
    } else {
      T[0] = Tt * (delta[0] / Dt);
      T[1] = Tt * (delta[1] / Dt);
      Dm[0] = dTtdDt * sq(delta[0] / Dt) + (Tt / Dt) * (1 - sq(delta[0] / Dt));
      Dm[1] = (dTtdDt - Tt / Dt) * (delta[0] * delta[1] / (Dt * Dt));
      Dm[2] = dTtdDn * (delta[0] / Dt);
      Dm[3] = (dTtdDt - Tt / Dt) * (delta[0] * delta[1] / (Dt * Dt));
      Dm[4] = dTtdDt * sq(delta[1] / Dt) + (Tt / Dt) * (1 - sq(delta[1] / Dt));
      Dm[5] = dTtdDn * (delta[1] / Dt);
      Dm[6] = dTndDt * (delta[0] / Dt);
      Dm[7] = dTndDt * (delta[1] / Dt);
      Dm[8] = dTndDn;
    }
    // zone from the larger of the normalised openings
    const double a = Dn / c.delta_cn, b = Dt / c.delta_ct;
    const double nf = (a > b) ? a : b;
    *zone = (nf <= 0) ? 0 : (nf <= 1 ? 1 : (nf <= 5.0 ? 2 : 3));
    return;
  }
  // bilinear and Ortiz-Pandolfi share the effective-opening form
  double deff = sq(delta[dim - 1]);
  for (int i = 0; i < dim - 1; ++i) deff += c.beta2 * sq(delta[i]);
  deff = sqrt(deff);
  double trac = 0.0, dtrac = 0.0;
  double dmax_copy = 0.0;
  double tl_c = 0.0;           // trilinear: compression-penalty coefficient
  if (law >= COH_TL) {
    // Trilinear laws.  The plain ones read delta_max but never write it (like the bilinear one),
    // and their max_traction is set only on the unloading branch, so a compressed point on the
    // loading branch with delta_max > 0 gets a zero penalty (src/Material_TrilinearCohesive.cpp:
    // 40-128, src/Material_SmoothedTrilinearCohesive.cpp:40-140).
    const bool smooth = (law == COH_STL || law == COH_STLNU);
    const bool memory = (law == COH_TL || law == COH_STL);
    const double delta_max = memory ? isv[0] : 0.0;
    double max_traction = 0.0;
    if (!memory || deff >= delta_max || deff < 0.0) {
      trilinear_curve(c, smooth, false, deff, &trac, &dtrac);
    } else {
      double unused;
      trilinear_curve(c, smooth, true, delta_max, &max_traction, &unused);
      trac = max_traction * (deff / delta_max);
      dtrac = max_traction / delta_max;
    }
    if (memory && delta_max > 0.0) tl_c = (max_traction / c.alpha) * (c.delta_c1 / delta_max);
    else tl_c = (smooth ? 2.0 * c.sigma_c : c.sigma_c) / c.alpha;
  } else if (law == COH_BL || law == COH_BLNU) {
    // BilinearCohesiveMaterial never writes delta_max, so both variants follow the loading curve.
    const double delta_max = (law == COH_BL) ? isv[0] : 0.0;
    if (law == COH_BLNU || deff >= delta_max || deff < 0.0) {
      if (deff >= 0 && deff < c.delta_c1) { trac = deff * (c.sigma_c / c.delta_c1); dtrac = (c.sigma_c / c.delta_c1); }
      else if (deff >= c.delta_c1 && deff < c.delta_c2) {
        trac = c.sigma_c * (1 - (deff - c.delta_c1) / (c.delta_c2 - c.delta_c1));
        dtrac = -1.0 * (c.sigma_c / (c.delta_c2 - c.delta_c1));
      } else { trac = 0; dtrac = 0; }
    } else {
      double max_traction;
      if (delta_max >= 0 && delta_max < c.delta_c1) max_traction = delta_max * (c.sigma_c / c.delta_c1);
      else if (delta_max >= c.delta_c1 && delta_max < c.delta_c2) max_traction = c.sigma_c * (1 - (delta_max - c.delta_c1) / (c.delta_c2 - c.delta_c1));
      else max_traction = 0;
      trac = max_traction * (deff / delta_max);
      dtrac = max_traction / delta_max;
    }
  } else {
    const bool unloading_law = (law == COH_OP || law == COH_OPAUG);
    if (unloading_law) {
      double& delta_max = isv[0];
      dmax_copy = delta_max;
      if (deff >= delta_max || deff < 0.0) {
        trac = c.sigma_c * (deff / c.delta_c) * exp(1.0 - deff / c.delta_c);
        dtrac = (c.sigma_c / c.delta_c) * (1.0 - deff / c.delta_c) * exp(1.0 - deff / c.delta_c);
        delta_max = deff;
      } else {
        const double max_traction = c.sigma_c * (delta_max / c.delta_c) * exp(1.0 - delta_max / c.delta_c);
        trac = max_traction * (deff / delta_max);
        dtrac = max_traction / delta_max;
      }
    } else {
      trac = c.sigma_c * (deff / c.delta_c) * exp(1.0 - deff / c.delta_c);
      dtrac = (c.sigma_c / c.delta_c) * (1.0 - deff / c.delta_c) * exp(1.0 - deff / c.delta_c);
    }
  }
  double br[3], dd[3];
  for (int i = 0; i < dim; ++i) br[i] = c.beta2 * delta[i];
  br[dim - 1] += (1.0 - c.beta2) * delta[dim - 1];
  for (int i = 0; i < dim; ++i) T[i] = (trac / deff) * br[i];
  const bool compress = delta[dim - 1] < 0;
  if (compress) {
    if (law == COH_OPAUG) T[dim - 1] = (c.sigma_c / c.alpha) * exp(1.0 - dmax_copy / c.delta_c) * sinh(c.alpha * delta[dim - 1] / c.delta_c);
    else if (law == COH_OPNUAUG) T[dim - 1] = (c.sigma_c * exp(1.0) / c.alpha) * sinh(c.alpha * delta[dim - 1] / c.delta_c);
  }
  dd[dim - 1] = delta[dim - 1] / deff;
  for (int i = 0; i < dim - 1; ++i) dd[i] = c.beta2 * delta[i] / deff;
  for (int i = 0; i < dim; ++i)
    for (int k = 0; k < dim; ++k)
      Dm[i * dim + k] = br[i] * (dtrac * deff - trac) * (dd[k] / sq(deff)) +
                        (trac / deff) * (c.beta2 * (i == k ? 1.0 : 0.0) + (1.0 - c.beta2) * (i == dim - 1 ? 1.0 : 0.0) * (k == dim - 1 ? 1.0 : 0.0));
  if (compress) {
    if (law == COH_BL || law == COH_BLNU) {
      T[dim - 1] = (c.sigma_c / c.alpha) * sinh(c.alpha * delta[dim - 1] / c.delta_c1);
      for (int i = 0; i < dim - 1; ++i) Dm[(dim - 1) * dim + i] = 0.0;
      Dm[(dim - 1) * dim + dim - 1] = (c.sigma_c / c.delta_c1) * cosh(c.alpha * delta[dim - 1] / c.delta_c1);
    } else if (law == COH_OPAUG) {
      for (int i = 0; i < dim - 1; ++i) Dm[(dim - 1) * dim + i] = 0.0;
      Dm[(dim - 1) * dim + dim - 1] = (c.sigma_c / c.delta_c) * exp(1.0 - dmax_copy / c.delta_c) * cosh(c.alpha * delta[dim - 1] / c.delta_c);
    } else if (law == COH_OPNUAUG) {
      for (int i = 0; i < dim - 1; ++i) Dm[(dim - 1) * dim + i] = 0.0;
      Dm[(dim - 1) * dim + dim - 1] = (c.sigma_c * exp(1.0) / c.delta_c) * cosh(c.alpha * delta[dim - 1] / c.delta_c);
    } else if (law >= COH_TL) {
      T[dim - 1] = tl_c * sinh(c.alpha * delta[dim - 1] / c.delta_c1);
      for (int i = 0; i < dim - 1; ++i) Dm[(dim - 1) * dim + i] = 0.0;
      Dm[(dim - 1) * dim + dim - 1] = tl_c * (c.alpha / c.delta_c1) * cosh(c.alpha * delta[dim - 1] / c.delta_c1);
    }
  }
  if (law == COH_BL || law == COH_BLNU) {
    *zone = compress ? 0 : (deff <= c.delta_c1 ? 1 : (deff <= c.delta_c2 ? 2 : 3));
  } else if (law >= COH_TL) {
    *zone = compress ? 0 : (deff <= c.delta_c1 ? 1 : (deff <= c.delta_c3 ? 2 : 3));
  } else {
    const double nf = deff / c.delta_c;
    *zone = (nf <= 0) ? 0 : (nf <= 1 ? 1 : (nf <= 5.0 ? 2 : 3));
  }
}

// The DIM components of a node-major array at `node` (coordinates, displacements): one 16-byte
// load in 2D (the arrays are 16-byte aligned; pg_assemble_device checks a caller's U), DIM loads
// in 3D.  Read-only for the whole kernel.
template <int DIM>
__device__ __forceinline__ void load_node(const double* __restrict__ A, int node, double* v) {
  if constexpr (DIM == 2) {
    const double2 t = __ldg(reinterpret_cast<const double2*>(A) + node);
    v[0] = t.x;
    v[1] = t.y;
  } else {
#pragma unroll
    for (int d = 0; d < DIM; ++d) v[d] = __ldg(&A[(size_t)node * DIM + d]);
  }
}

// Voigt B-matrix entry B(r, k*dim + q) for a node with gradient g (dim entries).
template <typename T>
__device__ inline T bmat(int dim, int r, int q, const T* g) {
  if (dim == 2) {
    if (r == 0) return q == 0 ? g[0] : T(0);
    if (r == 1) return q == 1 ? g[1] : T(0);
    return q == 0 ? g[1] : g[0];
  }
  switch (r) {
    case 0: return q == 0 ? g[0] : T(0);
    case 1: return q == 1 ? g[1] : T(0);
    case 2: return q == 2 ? g[2] : T(0);
    case 3: return q == 0 ? T(0) : (q == 1 ? g[2] : g[1]);
    case 4: return q == 1 ? T(0) : (q == 0 ? g[2] : g[0]);
    default: return q == 2 ? T(0) : (q == 0 ? g[1] : g[0]);
  }
}

}  // namespace pgd
