// pg_setup.h -- host-side IGFEM set-up for the B200 assembly path.
//
// Builds, once per mesh, everything the device assembly consumes: the structured background
// mesh, inclusion detection, the cut-case tables of the cut elements, enrichment (and cohesive
// mirror) nodes, the sub-element and cohesive quadrature data of the cut elements, the global DOF
// numbering and the CSR pattern of the four PETSc-style blocks (ff, fp, pf, pp).  Each step
// restates the reference algorithm it replaces; the citations are in pg_setup.cpp.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace pg {

enum ElemType : int { TRI3 = 0, QUAD4 = 1, TET4 = 2 };
enum SubType : int { SUB_TRI3 = 0, SUB_QUAD4 = 1, SUB_POLYGON = 2, SUB_TET4 = 3, SUB_PRISM6 = 4, SUB_HEX8 = 5 };
enum CohLaw : int {
  COH_NONE = 0, COH_BL = 1, COH_BLNU = 2, COH_XN = 3, COH_XNNU = 4,
  COH_OP = 5, COH_OPNU = 6, COH_OPAUG = 7, COH_OPNUAUG = 8,
  COH_TL = 9, COH_TLNU = 10, COH_STL = 11, COH_STLNU = 12
};

// Problem description (the reference's Tests/Main.cpp inputs).
struct ProblemDesc {
  int elem_type = TRI3;
  int n[3] = {8, 8, 0};
  double lo[3] = {0, 0, 0};
  double hi[3] = {1, 1, 0};
  std::vector<double> incl;  // circles (cx, cy, r) or spheres (cx, cy, cz, r)
  double E_matrix = 3.5e3, nu_matrix = 0.35, E_fiber = 72e3, nu_fiber = 0.22;
  int coh_law = COH_NONE;
  double coh[4] = {0, 0, 0, 0};
  int plane_strain = 1;
  int subscale = 0;
  double eps_macro[6] = {0, 0, 0, 0, 0, 0};
  double app_strain = 0.0;
  double ply_frac = 0.0;     // bounding plies: fraction of the height at the top and the bottom
  double ply[5] = {0, 0, 0, 0, 0};   // E1, E2, G12, G23, nu12 of the plies
};

// Cohesive-law constants as the reference's materials hold them after set_parameter.
struct CohParams {
  int law = COH_NONE;
  int nvar = 0;  // internal variables per cohesive quadrature point
  double sigma_c = 0, delta_c1 = 0, delta_c2 = 0;  // bilinear (and trilinear)
  double delta_c3 = 0;                             // trilinear
  double delta_cn = 0, delta_ct = 0, q = 0;        // Xu-Needleman
  double delta_c = 0;                              // Ortiz-Pandolfi
  double beta2 = 1.0, alpha = 50.0;
};

struct Setup {
  ProblemDesc desc;
  int dim = 2;
  int etype = TRI3;
  int npe = 3;  // nodes per parent element
  bool cohesive = false;
  CohParams coh;
  // materials: 0 = matrix, 1 = fiber (linear elastic isotropic), 2 = bounding plies (linear
  // elastic transversely isotropic); D in Voigt order, row-major
  int nvoigt = 3;
  double D[3][36];
  // derivatives of D of materials 0 and 1 by E, lambda, mu, K and nu, as
  // LinearElasticIsotropicMaterial::computeDmatSensitivities forms them (material sensitivities)
  double dD[2][5][36];

  // nodes: standard nodes first, then enrichment nodes (cohesive mirrors after the originals)
  int n_std = 0, n_enr = 0, n_enr_initial = 0;
  std::vector<double> X;         // (n_std + n_enr) * dim
  std::vector<int> node_detect;  // per standard node: inclusion index or -1
  std::vector<int> dnode;        // node -> node that owns its DOFs (periodic primary), per node
  std::vector<int> enr_edge;     // per enrichment node: 2 standard node ids (sorted)
  std::vector<int> enr_incl;     // per enrichment node: inclusion index

  // elements
  int ne = 0;
  std::vector<int> conn;      // ne * npe
  std::vector<int> elem_mat;  // 0 matrix / 1 fiber (uncut elements)
  std::vector<int> cut_of;    // element -> cut index or -1

  // cut elements
  int ncut = 0;
  std::vector<int> cut_elem;                  // cut index -> element
  std::vector<int> cut_node_off, cut_nodes;   // parent nodes then enrichment nodes (global node ids)
  std::vector<int> cut_sub_off, sub_type, sub_mat, sub_node_off, sub_nodes;  // sub-elements (global node ids)
  std::vector<int> sub_qp_off;  // first quadrature point of each sub-element (into qp_wgt)
  std::vector<int> cut_qp_off;                // volumetric quadrature points per cut element
  std::vector<double> qp_wgt;                 // J * W of each volumetric qp
  std::vector<int> qp_mat;                    // material of each qp
  std::vector<int> qp_grad_off;               // offset (in doubles) of each qp's gradient block
  std::vector<double> qp_grad;                // n_nodes_of_cut_elem * dim per qp
  std::vector<int> cut_coh_off;               // cohesive elements per cut element
  std::vector<int> coh_nh;                    // nodes per side of each cohesive element
  std::vector<int> coh_local_off, coh_local;  // local indices (into the cut element's node list): '-' side then '+' side
  std::vector<int> coh_qp_off;                // qps per cohesive element
  std::vector<double> cqp_N;                  // nh per qp
  std::vector<double> cqp_R;                  // dim*dim per qp (rows: tangent(s), normal)
  std::vector<double> cqp_wgt;                // J * W
  std::vector<int> cqp_isv;                   // offset of the qp's internal variables in the ISV array
  int n_isv = 0;

  // DOFs
  int n_free = 0, n_const = 0;
  std::vector<int> node_dof;  // per node (incl. enrichment) * dim: global DOF (free < n_free <= constrained)
  std::vector<double> dirichlet;  // per constrained DOF (index - n_free): prescribed value at t_frac = 1

  // CSR pattern of K split into ff / fp / pf / pp (columns sorted), exactly the locations the
  // reference's Assembler::set_matrix inserts.
  std::vector<int> rp[4], ci[4];
  int nrows[4] = {0, 0, 0, 0}, ncols[4] = {0, 0, 0, 0};

  // Row-owner structures: rows of K are owned by "DOF nodes" (nodes that own DOFs).
  int n_dn = 0;                        // number of DOF nodes
  std::vector<int> dn_node;            // DOF node -> node id
  std::vector<int> node_dn;            // node -> DOF node (via dnode)
  std::vector<int> dn_nbr_off, dn_nbr; // sorted neighbour DOF nodes
  std::vector<int> dn_adj_off, dn_adj; // adjacent (element, local node) pairs: elem * 32 + local

  std::string error;
};

// Results of the device preprocessing passes (pg_prep.cu) for a structured mesh, consumed by
// build_setup in place of its own loops.  Every table equals what build_setup forms itself.
struct PrepResult {
  bool valid = false;
  std::vector<int> node_detect;         // per standard node: inclusion index or -1
  int surface_node = -1;                // first node on an inclusion surface, or -1
  std::vector<unsigned char> elem_flag; // 0 uncut (own material), 1 inside an inclusion, 2 cut candidate
  bool edges_valid = false;             // the enrichment nodes below are the set-up's (tri3, or one inclusion per element)
  std::vector<int> enr_edge, enr_incl;  // per enrichment node (mirrors not included): sorted node pair, inclusion
  std::vector<double> XE;               // per enrichment node: 3 coordinates
  int no_sign_change = -1;              // first enrichment node whose edge has no sign change, or -1
  std::vector<int> std_dof;             // standard node * dim: free index >= 0, or -1 - (constrained index)
  bool pattern_on_device = false;       // build_setup leaves the adjacency and the pattern to device_pattern
  double device_ms = 0.0;               // device time of the passes
};

// Runs the device passes of pg_prep.cu; 0 on success (pr.valid false when the mesh is outside
// what they cover), nonzero with err set when a CUDA call fails.
int device_prep(const ProblemDesc& d, PrepResult& pr, std::string& err);

// The DOF nodes' adjacency and neighbour lists and the CSR pattern of the four blocks, from the
// rest of the set-up: on the host (build_pattern) or on the device (device_pattern, pg_prep.cu;
// the same tables bit for bit).  0 on success; device_pattern returns nonzero with err set when a
// CUDA call fails, build_pattern with Setup::error set when the mesh is too large.
int build_pattern(Setup& s);
int device_pattern(Setup& s, std::string& err, double* device_ms);

// Returns 0 on success, a nonzero status with Setup::error filled otherwise.  pr (optional, valid)
// supplies the node detection, the element pass, the enrichment nodes and the standard nodes' DOF
// numbering from the device.
int build_setup(const ProblemDesc& d, Setup& s, const PrepResult* pr = nullptr);

}  // namespace pg
