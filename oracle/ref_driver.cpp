/*
 * ref_driver.cpp -- C entry points around the reference PIGFEM classes, compiled and linked
 * together with the reference's own sources into oracle/_ref/libpigfem_ref.so.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product links this.  It lets the parity tests and
 * the CPU-baseline leg of bench.py:
 *   - build a problem the way Tests/Main.cpp:150-648 does (structured mesh from
 *     Mesh::generate_mesh, circular or spherical inclusions, linear-elastic matrix and fiber,
 *     an optional cohesive law on every fiber/matrix interface, Dirichlet strain or subscale
 *     loading),
 *   - run Problem::init / Problem::setup (IGFEM detection, enrichment, Mesh::store_shape_functions,
 *     DOF numbering, CSR preallocation),
 *   - call Assembler::assemble (src/Assembler.cpp:65-146) on a caller-given displacement vector
 *     and committed internal variables and read back K (ff, fp, pf, pp), P_int (f, p) and the
 *     trial internal variables,
 *   - run the reference's own nonlinear solve (SolverNonlinear::solve, src/SolverNonlinear.cpp:70)
 *     and return its Newton log,
 *   - export the enriched mesh (coordinates, element/enrichment topology, per-quadrature-point
 *     shape data, DOF map) so the product's own preprocessing can be checked against it.
 * Protected/private members are reached by redefining the access keywords for this one TU.
 */
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <iomanip>
#include <iostream>
#include <iterator>
#include <limits>
#include <map>
#include <numeric>
#include <set>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>
#include <chrono>

#include "../include/pigfem_b200_dropin.h"
// Defined only when the drop-in Assembler::assemble and libpigfem_b200.so are linked in.
extern "C" int pg_dropin_bind(void* problem, const pg_problem_desc* desc) __attribute__((weak));
extern "C" const char* pg_dropin_last_error(void) __attribute__((weak));
#include <sys/time.h>
#include <unistd.h>

#define protected public
#define private public
#include "Mesh.h"
#include "Problem.h"
#include "ProblemLinearElasticity.h"
#include "ProblemNonlinearStructural.h"
#include "Solver.h"
#include "Assembler.h"
#include "DofObject.h"
#include "NodalData.h"
#include "InternalVars.h"
#include "BoundaryObject.h"
#include "elem.h"
#include "CohesiveElem.h"
#include "material_lei.h"
#include "material_leti.h"
#include "Material_BilinearCohesive.h"
#include "Material_BilinearCohesiveNU.h"
#include "Material_XNCohesive.h"
#include "Material_XNCohesiveNU.h"
#include "Material_OPCohesive.h"
#include "Material_OPCohesiveNU.h"
#include "Material_OPCohesiveAug.h"
#include "Material_OPCohesiveNUAug.h"
#include "Material_TrilinearCohesive.h"
#include "Material_TrilinearCohesiveNU.h"
#include "Material_SmoothedTrilinearCohesive.h"
#include "Material_SmoothedTrilinearCohesiveNU.h"
#include "InclusionCircle.h"
#include "InclusionSphere.h"
#include "Options.h"
#include "Utilities.h"
#include "CohesiveElem.h"
#include "pgshim_objects.h"
#include "WriterHomogenization.h"
#include "SensitivitySolver.h"
#include "SensitivityParameter.h"
#include "SensitivityRightLoad.h"
#undef protected
#undef private

extern bool writeToScreen;
extern std::string logFile;

extern "C" {

/* Cohesive-law selectors (Tests/Main.cpp:370-390 choices, plus the plain and NU variants). */
enum {
  PGREF_COH_NONE = 0,
  PGREF_COH_BL = 1,      /* BilinearCohesiveMaterial:  SIGMA_C, DELTA_C1, DELTA_C2 */
  PGREF_COH_BLNU = 2,    /* BilinearCohesiveNUMaterial */
  PGREF_COH_XN = 3,      /* XNCohesiveMaterial:        SIGMA_C, DELTA_CN, DELTA_CT, Q */
  PGREF_COH_XNNU = 4,    /* XNCohesiveNUMaterial */
  PGREF_COH_OP = 5,      /* OPCohesiveMaterial:        SIGMA_C, DELTA_C, BETA */
  PGREF_COH_OPNU = 6,    /* OPCohesiveNUMaterial */
  PGREF_COH_OPAUG = 7,   /* OPCohesiveAugMaterial */
  PGREF_COH_OPNUAUG = 8, /* OPCohesiveNUAugMaterial */
  PGREF_COH_TL = 9,      /* TrilinearCohesiveMaterial: SIGMA_C, DELTA_C1, DELTA_C2, DELTA_C3 */
  PGREF_COH_TLNU = 10,   /* TrilinearCohesiveNUMaterial */
  PGREF_COH_STL = 11,    /* TrilinearSmoothedCohesiveMaterial */
  PGREF_COH_STLNU = 12   /* TrilinearSmoothedCohesiveNUMaterial */
};

typedef struct {
  int elem_type;              /* 0 = TRI3, 1 = QUAD4, 2 = TET4 */
  int nx, ny, nz;
  double xmin, xmax, ymin, ymax, zmin, zmax;
  int n_incl;
  const double* incl;         /* circles: cx, cy, r ; spheres: cx, cy, cz, r */
  double E_matrix, nu_matrix, E_fiber, nu_fiber;
  int coh_law;
  double coh[4];              /* law parameters in the order listed above */
  int plane_strain;
  int subscale;               /* 1: periodic mesh + macroscale strain eps_macro, node 0 pinned */
  double eps_macro[6];
  double app_strain;          /* Dirichlet mode: right x = app_strain*(xmax-xmin), left x = 0, node 0 pinned */
  double ply_frac;            /* bounding plies: top / bottom fraction of the height (0: none) */
  double ply[5];              /* ply material E1, E2, G12, G23, nu12 */
  int sens_mat;               /* material sensitivity: 0 none, 1 "Matrix", 2 "Fiber" */
  int sens_param;             /* 0 E, 1 LAMBDA, 2 MU, 3 K, 4 NU */
} pgref_config;

}  // extern "C"

namespace {

struct Export {
  std::vector<int> i32;
  std::vector<double> f64;
  bool is_int = true;
};

struct Handle {
  int argc = 1;
  char arg0[8] = "oracle";
  char* argv_store[2] = {arg0, nullptr};
  char** argv = argv_store;
  Mesh* mesh = nullptr;
  Problem* prob = nullptr;
  LinearElasticIsotropicMaterial* fiber = nullptr;
  std::vector<Inclusion*> incs;
  bool nonlinear = false;
  std::map<std::string, Export> out;
  std::string log_path;
  std::string err;
  pgref_config cfg{};            // the configuration it was built from (incl points into incl_store)
  std::vector<double> incl_store;
};

Export& put_i(Handle* h, const std::string& k) { Export& e = h->out[k]; e.is_int = true; e.i32.clear(); return e; }
Export& put_d(Handle* h, const std::string& k) { Export& e = h->out[k]; e.is_int = false; e.f64.clear(); return e; }

void export_mat(Handle* h, const std::string& name, Mat A) {
  Export& rp = put_i(h, name + "_rowptr");
  Export& ci = put_i(h, name + "_cols");
  Export& v = put_d(h, name + "_vals");
  rp.i32.push_back(0);
  for (int i = 0; i < A->m; ++i) {
    for (size_t k = 0; k < A->cols[i].size(); ++k) { ci.i32.push_back(A->cols[i][k]); v.f64.push_back(A->vals[i][k]); }
    rp.i32.push_back((int)ci.i32.size());
  }
  Export& sh = put_i(h, name + "_shape");
  sh.i32 = {A->m, A->n};
}

void export_vec(Handle* h, const std::string& name, Vec x) { put_d(h, name).f64 = x->a; }

Material* make_cohesive(int law, const double* p) {
  Material* m = nullptr;
  switch (law) {
    case PGREF_COH_BL: m = new BilinearCohesiveMaterial; break;
    case PGREF_COH_BLNU: m = new BilinearCohesiveNUMaterial; break;
    case PGREF_COH_XN: m = new XNCohesiveMaterial; break;
    case PGREF_COH_XNNU: m = new XNCohesiveNUMaterial; break;
    case PGREF_COH_OP: m = new OPCohesiveMaterial; break;
    case PGREF_COH_OPNU: m = new OPCohesiveNUMaterial; break;
    case PGREF_COH_OPAUG: m = new OPCohesiveAugMaterial; break;
    case PGREF_COH_OPNUAUG: m = new OPCohesiveNUAugMaterial; break;
    case PGREF_COH_TL: m = new TrilinearCohesiveMaterial; break;
    case PGREF_COH_TLNU: m = new TrilinearCohesiveNUMaterial; break;
    case PGREF_COH_STL: m = new TrilinearSmoothedCohesiveMaterial; break;
    case PGREF_COH_STLNU: m = new TrilinearSmoothedCohesiveNUMaterial; break;
    default: return nullptr;
  }
  m->set_name("Interface");
  if (law == PGREF_COH_BL || law == PGREF_COH_BLNU) {
    m->set_parameter("SIGMA_C", p[0]); m->set_parameter("DELTA_C1", p[1]); m->set_parameter("DELTA_C2", p[2]);
  } else if (law >= PGREF_COH_TL) {
    m->set_parameter("SIGMA_C", p[0]); m->set_parameter("DELTA_C1", p[1]); m->set_parameter("DELTA_C2", p[2]);
    m->set_parameter("DELTA_C3", p[3]);
  } else if (law == PGREF_COH_XN || law == PGREF_COH_XNNU) {
    m->set_parameter("SIGMA_C", p[0]); m->set_parameter("DELTA_CN", p[1]); m->set_parameter("DELTA_CT", p[2]); m->set_parameter("Q", p[3]);
  } else {
    m->set_parameter("SIGMA_C", p[0]); m->set_parameter("DELTA_C", p[1]); m->set_parameter("BETA", p[2]);
  }
  return m;
}

// The enriched mesh, DOF map and per-quadrature-point data consumed by Assembler::assemble.
void export_mesh(Handle* h) {
  Mesh* mesh = h->mesh;
  DofObject* dofs = h->prob->get_dofs();
  const int dim = (int)mesh->dim();
  Export& nc = put_d(h, "node_coords");
  for (id_type n = 0; n < mesh->n_local_nodes(); ++n) {
    Node* nd = mesh->_nodes[n];
    for (int d = 0; d < dim; ++d) nc.f64.push_back((*nd)(d));
  }
  Export& ec = put_d(h, "enrich_coords");
  Export& eid = put_i(h, "enrich_ids");
  for (id_type n = 0; n < mesh->n_local_enrich_nodes(); ++n) {
    Node* nd = mesh->get_enrich_node(n);
    for (int d = 0; d < dim; ++d) ec.f64.push_back((*nd)(d));
    eid.i32.push_back((int)(nd->get_id() - ENRICH_START));
  }
  // node-major DOF map: standard nodes, then enrichment nodes (local order)
  Export& dm = put_i(h, "node_dofs");
  for (id_type n = 0; n < mesh->n_local_nodes() + mesh->n_local_enrich_nodes(); ++n) {
    id_type idx = n < mesh->n_local_nodes() ? n : ENRICH_START + (n - mesh->n_local_nodes());
    std::vector<id_type>& g = dofs->get_nodal_global_dofs_local(idx);
    for (int d = 0; d < dim; ++d) dm.i32.push_back(d < (int)g.size() ? (int)g[d] : -1);
  }
  put_i(h, "n_free_const").i32 = {(int)dofs->n_global_free_dofs(), (int)dofs->n_global_const_dofs()};

  Export& eoff = put_i(h, "elem_node_off");
  Export& enodes = put_i(h, "elem_nodes");     // standard nodes then enrichment nodes (id - ENRICH_START + n_nodes_total)
  Export& ecut = put_i(h, "elem_cut");
  Export& edof_off = put_i(h, "elem_dof_off");
  Export& edofs = put_i(h, "elem_dofs");
  Export& qoff = put_i(h, "elem_qp_off");       // volumetric qps per element
  Export& qgrad = put_d(h, "qp_grad");          // per volumetric qp: (n_nodes_e x dim)
  Export& qgoff = put_i(h, "qp_grad_off");
  Export& qJ = put_d(h, "qp_J");
  Export& qW = put_d(h, "qp_W");
  Export& qmat = put_i(h, "qp_mat");            // material index (mesh order) of the qp
  Export& coff = put_i(h, "elem_coh_off");      // cohesive elements per element
  Export& cstruct = put_i(h, "coh_struct");     // per cohesive element: local node indices into the element's node list
  Export& cstruct_off = put_i(h, "coh_struct_off");
  Export& cqoff = put_i(h, "coh_qp_off");       // qps per cohesive element
  Export& cN = put_d(h, "coh_qp_N");
  Export& cNoff = put_i(h, "coh_qp_N_off");
  Export& cR = put_d(h, "coh_qp_R");            // dim x dim per qp
  Export& cJ = put_d(h, "coh_qp_J");
  Export& cW = put_d(h, "coh_qp_W");
  Export& cmat = put_i(h, "coh_mat");
  Export& esub_off = put_i(h, "elem_sub_off");
  Export& esub_type = put_i(h, "sub_type");
  Export& esub_nodes_off = put_i(h, "sub_nodes_off");
  Export& esub_nodes = put_i(h, "sub_nodes");   // local node indices of each integration element
  Export& esub_mat = put_i(h, "sub_mat");
  eoff.i32.push_back(0); edof_off.i32.push_back(0); qoff.i32.push_back(0); qgoff.i32.push_back(0);
  coff.i32.push_back(0); cstruct_off.i32.push_back(0); cqoff.i32.push_back(0); cNoff.i32.push_back(0);
  esub_off.i32.push_back(0); esub_nodes_off.i32.push_back(0);
  const id_type n_std = mesh->n_local_nodes();
  std::map<Material*, int> mat_index;
  for (size_t m = 0; m < mesh->_materials.size(); ++m) mat_index[mesh->_materials[m]] = (int)m;
  for (Mesh::element_iterator it = mesh->active_elements_begin(); it != mesh->active_elements_end(); ++it) {
    Elem* el = *it;
    id_type l_elem = mesh->global_to_local_elem(el->get_id());
    for (id_type n = 0; n < el->n_nodes(); ++n) enodes.i32.push_back((int)el->get_node(n)->get_id());
    for (id_type n = 0; n < el->n_enrich_nodes(); ++n) enodes.i32.push_back((int)(el->get_enrich_node(n)->get_id() - ENRICH_START + n_std));
    eoff.i32.push_back((int)enodes.i32.size());
    ecut.i32.push_back(el->is_intersected() ? 1 : 0);
    std::vector<id_type> ed;
    dofs->get_elem_global_dofs(el, ed);
    for (id_type d : ed) edofs.i32.push_back((int)d);
    edof_off.i32.push_back((int)edofs.i32.size());
    id_type nvq = mesh->n_volumetric_qps(l_elem);
    for (id_type q = 0; q < nvq; ++q) {
      std::vector<std::vector<double>>& g = mesh->get_shape_grad(l_elem, q);
      for (auto& row : g) for (double v : row) qgrad.f64.push_back(v);
      qgoff.i32.push_back((int)qgrad.f64.size());
      qJ.f64.push_back(mesh->get_J(l_elem, q));
      qW.f64.push_back(mesh->get_W(l_elem, q));
    }
    if (!el->is_intersected()) {
      Material* m = mesh->get_element_material_global(el->get_id());
      for (id_type q = 0; q < nvq; ++q) qmat.i32.push_back(mat_index[m]);
    } else {
      for (id_type ie = 0; ie < el->n_integration_elem(); ++ie) {
        Material* m = mesh->get_element_material_global(el->get_id(), ie);
        Elem* sub = el->get_integration_elem(ie);
        for (id_type q = 0; q < sub->n_q_points(); ++q) qmat.i32.push_back(mat_index[m]);
        esub_type.i32.push_back((int)sub->get_type());
        esub_mat.i32.push_back(mat_index[m]);
      }
      std::vector<std::vector<short_id_type>>& st = el->_int_elem_struct;
      (void)st;
    }
    esub_off.i32.push_back((int)esub_type.i32.size());
    qoff.i32.push_back((int)qJ.f64.size());
    if (mesh->is_cohesive() && el->is_intersected()) {
      std::vector<std::vector<short_id_type>>& cs = el->getCohesiveElemStructure();
      id_type curr_qp = nvq;
      for (id_type ce = 0; ce < el->n_cohesive_elem(); ++ce) {
        for (short_id_type v : cs[ce]) cstruct.i32.push_back((int)v);
        cstruct_off.i32.push_back((int)cstruct.i32.size());
        CohesiveElem* c = el->get_cohesive_elem(ce);
        cmat.i32.push_back(mat_index[el->get_cohesive_material(ce)]);
        for (id_type q = 0; q < c->n_q_points(); ++q) {
          std::vector<double>& N = mesh->get_shape(l_elem, curr_qp);
          for (double v : N) cN.f64.push_back(v);
          cNoff.i32.push_back((int)cN.f64.size());
          DenseMatrix<double>& R = mesh->get_rot_matrix(l_elem, curr_qp);
          for (id_type a = 0; a < R.n_rows(); ++a) for (id_type b = 0; b < R.n_cols(); ++b) cR.f64.push_back(R(a, b));
          cJ.f64.push_back(mesh->get_J(l_elem, curr_qp));
          cW.f64.push_back(mesh->get_W(l_elem, curr_qp));
          curr_qp++;
        }
        cqoff.i32.push_back((int)cJ.f64.size());
      }
    }
    coff.i32.push_back((int)cmat.i32.size());
  }
  (void)esub_nodes; (void)esub_nodes_off;
  Export& mats = put_d(h, "materials");  // per material: kind (0 lei, 1 cohesive, 2 leti), E (E1), nu (nu12)
  for (Material* m : mesh->_materials) {
    if (m->is_cohesive()) { mats.f64.push_back(1); mats.f64.push_back(0); mats.f64.push_back(0); }
    else if (dynamic_cast<LinearElasticTransverselyIsotropicMaterial*>(m)) {
      mats.f64.push_back(2); mats.f64.push_back(m->get_parameter("E1")); mats.f64.push_back(m->get_parameter("NU12"));
    }
    else { mats.f64.push_back(0); mats.f64.push_back(m->get_parameter("E")); mats.f64.push_back(m->get_parameter("nu")); }
  }
  // internal-variable layout: per element, per qp, count
  Export& isv_off = put_i(h, "isv_off");
  isv_off.i32.push_back(0);
  InternalVars* iv = h->prob->get_internal_vars();
  std::vector<std::vector<std::vector<double>>>& all = iv->get_all_internal_vars();
  int run = 0;
  for (auto& e : all) for (auto& q : e) { run += (int)q.size(); isv_off.i32.push_back(run); }
  Export& isv_elem_off = put_i(h, "isv_elem_qp_off");
  isv_elem_off.i32.push_back(0);
  int qrun = 0;
  for (auto& e : all) { qrun += (int)e.size(); isv_elem_off.i32.push_back(qrun); }
}

}  // namespace

extern "C" {

void* pgref_create(const pgref_config* cfg) {
  Handle* h = new Handle;
  h->cfg = *cfg;
  h->incl_store.assign(cfg->incl, cfg->incl + (size_t)cfg->n_incl * ((cfg->elem_type == 2) ? 4 : 3));
  h->cfg.incl = h->incl_store.data();
  char tmpl[] = "/tmp/pgref_log_XXXXXX";
  int fd = mkstemp(tmpl);
  if (fd >= 0) close(fd);
  h->log_path = tmpl;
  h->mesh = new Mesh(&h->argc, &h->argv);
  Mesh& mesh = *h->mesh;
  mesh.init();
  h->nonlinear = cfg->coh_law != PGREF_COH_NONE;
  if (h->nonlinear) h->prob = new ProblemNonlinearStructural;
  else h->prob = new ProblemLinearElasticity;
  writeToScreen = false;
  logFile = h->log_path;
  h->prob->getOptions()->setBoolOption("-WRITE_VTK", "false");
  h->prob->set_parameter("plane_strain", cfg->plane_strain ? 1.0 : 0.0);
  h->prob->attach_mesh(&mesh);
  writeToScreen = false;
  logFile = h->log_path;

  const int dim = (cfg->elem_type == 2) ? 3 : 2;
  h->fiber = new LinearElasticIsotropicMaterial;
  h->fiber->set_parameter("E", cfg->E_fiber);
  h->fiber->set_parameter("nu", cfg->nu_fiber);
  h->fiber->set_name("Fiber");
  for (int i = 0; i < cfg->n_incl; ++i) {
    const double* v = cfg->incl + (size_t)i * (dim + 1);
    if (dim == 2) {
      Circle_Inclusion c;
      c.set_material(h->fiber);
      std::vector<double> ctr{v[0], v[1]};
      c.set_vec_parameter("center", ctr);
      c.set_parameter("r", v[2]);
      mesh.add_inclusion(&c);
    } else {
      Sphere_Inclusion s;
      s.set_material(h->fiber);
      std::vector<double> ctr{v[0], v[1], v[2]};
      s.set_vec_parameter("center", ctr);
      s.set_parameter("r", v[3]);
      mesh.add_inclusion(&s);
    }
  }
  if (cfg->subscale) mesh.set_periodic(true);
  if (cfg->elem_type == 0) mesh.generate_mesh(TRI3, cfg->xmin, cfg->xmax, cfg->nx, cfg->ymin, cfg->ymax, cfg->ny);
  else if (cfg->elem_type == 1) mesh.generate_mesh(QUAD4, cfg->xmin, cfg->xmax, cfg->nx, cfg->ymin, cfg->ymax, cfg->ny);
  else mesh.generate_mesh(TET4, cfg->xmin, cfg->xmax, cfg->nx, cfg->ymin, cfg->ymax, cfg->ny, cfg->zmin, cfg->zmax, cfg->nz);

  LinearElasticIsotropicMaterial matrix;
  matrix.set_parameter("E", cfg->E_matrix);
  matrix.set_parameter("nu", cfg->nu_matrix);
  matrix.set_name("Matrix");
  mesh.add_material(&matrix);
  mesh.set_material("Matrix");
  if (cfg->ply_frac > 0.0) {
    // bounding plies as Tests/Main.cpp:262-289 and 343-360 build them: element sets of the
    // elements whose nodes all lie in the top / bottom fraction of the height, given a linear
    // elastic transversely isotropic material
    std::set<id_type> top_ply, bottom_ply;
    const double y_lims = cfg->ymax - cfg->ymin;
    const double top_limit = cfg->ymax - y_lims * cfg->ply_frac;
    const double bottom_limit = cfg->ymin + y_lims * cfg->ply_frac;
    for (Mesh::element_iterator it = mesh.active_elements_begin(), end = mesh.active_elements_end(); it != end; ++it) {
      bool in_top_ply = true, in_bottom_ply = true;
      for (id_type n = 0; n < (*it)->n_nodes(); ++n) {
        std::vector<double> coords = (*it)->get_node(n)->get_coords();
        if (coords[1] < top_limit) in_top_ply = false;
        if (coords[1] > bottom_limit) in_bottom_ply = false;
      }
      if (in_top_ply) top_ply.insert((*it)->get_id());
      if (in_bottom_ply) bottom_ply.insert((*it)->get_id());
    }
    mesh.add_elemset("top_ply", top_ply);
    mesh.add_elemset("bottom_ply", bottom_ply);
    LinearElasticTransverselyIsotropicMaterial bounds;
    bounds.set_parameter("E1", cfg->ply[0]);
    bounds.set_parameter("E2", cfg->ply[1]);
    bounds.set_parameter("G12", cfg->ply[2]);
    bounds.set_parameter("G23", cfg->ply[3]);
    bounds.set_parameter("NU12", cfg->ply[4]);
    bounds.set_name("0_degree_plies");
    mesh.add_material(&bounds);
    mesh.set_material_from_elemset("0_degree_plies", "top_ply");
    mesh.set_material_from_elemset("0_degree_plies", "bottom_ply");
  }
  if (h->nonlinear) {
    Material* coh = make_cohesive(cfg->coh_law, cfg->coh);
    mesh.add_material(coh);
    delete coh;
  }
  BoundaryObject* boundary = h->prob->get_boundary();
  if (cfg->subscale) {
    std::vector<double> load(dim == 2 ? 3 : 6);
    for (size_t k = 0; k < load.size(); ++k) load[k] = cfg->eps_macro[k];
    h->prob->setMacroscaleValue(load);
    for (int d = 0; d < dim; ++d) boundary->set_dirichlet_bc(0, d, 0.0);
  } else {
    double app = (cfg->xmax - cfg->xmin) * cfg->app_strain;
    boundary->set_dirichlet_bcs_from_nodeset("right", 0, app);
    boundary->set_dirichlet_bcs_from_nodeset("left", 0, 0.0);
    for (int d = 0; d < dim; ++d) boundary->set_dirichlet_bc(0, d, 0.0);
  }
  if (cfg->sens_mat > 0) {
    // one material sensitivity parameter and the right-edge load function, as Tests/Main.cpp:586-609
    // registers them before Problem::init (which builds the sensitivity solver)
    static const char* params[5] = {"E", "LAMBDA", "MU", "K", "NU"};
    SensitivityRightLoad function;
    h->prob->addSensitivityFunction(&function);
    h->prob->addMaterialSensitivityParameter(cfg->sens_mat == 1 ? "Matrix" : "Fiber", params[cfg->sens_param]);
  }
  h->prob->init();
  h->prob->setup();
  export_mesh(h);
  return h;
}

/*
 * The reference's assemble_dPdd of the registered material parameter at the full DOF vector U
 * (free then constrained): exports dP_f and dP_p.  Returns 0, or -1 without a parameter.
 */
int pgref_sensitivity(void* vh, const double* U) {
  Handle* h = (Handle*)vh;
  if (h->cfg.sens_mat <= 0 || !h->prob->_sensitivity_solver || h->prob->_sensitivity_solver->_parameters.empty())
    return -1;
  writeToScreen = false;
  logFile = h->log_path;
  Solver* s = h->prob->get_solver();
  DofObject* dofs = h->prob->get_dofs();
  const int nf = (int)dofs->n_global_free_dofs(), np = (int)dofs->n_global_const_dofs();
  for (int i = 0; i < nf; ++i) s->_U.f->a[i] = U[i];
  for (int i = 0; i < np; ++i) s->_U.p->a[i] = U[nf + i];
  s->store_solution(s->_U, h->prob->get_solution());
  pvector dP;
  VecDuplicate(s->_U.f, &dP.f);
  VecDuplicate(s->_U.p, &dP.p);
  VecSet(dP.f, 0.0);
  VecSet(dP.p, 0.0);
  h->prob->_sensitivity_solver->_parameters[0]->assemble_dPdd(dP, h->prob);
  export_vec(h, "dP_f", dP.f);
  export_vec(h, "dP_p", dP.p);
  VecDestroy(&dP.f);
  VecDestroy(&dP.p);
  return 0;
}

/* Solver parameters as Tests/Main.cpp:627-632 sets them. */
void pgref_set_solver(void* vh, double rel_tol, double abs_tol, double max_dt, double min_dt, double T_final, int max_iter) {
  Handle* h = (Handle*)vh;
  Solver* s = h->prob->get_solver();
  s->set_dparameter("rel_tol", rel_tol);
  s->set_dparameter("abs_tol", abs_tol);
  s->set_dparameter("max_time_step", max_dt);
  s->set_dparameter("min_time_step", min_dt);
  s->set_dparameter("T_final", T_final);
  s->set_iparameter("max_iter", max_iter);
}

/*
 * One Assembler::assemble call.  U: full DOF vector (free then constrained, length
 * n_free + n_const).  isv_committed: flat committed internal variables in isv_off layout (may be
 * null: keep the current ones).  t_frac: load fraction (sets the macroscale strain for subscale
 * problems through Assembler::assemble_new_load_step).  Exports K_ff/K_fp/K_pf/K_pp, P_f, P_p and
 * isv_trial.  Returns the elapsed seconds of the assemble call alone.
 */
double pgref_assemble(void* vh, const double* U, const double* isv_committed, double t_frac, int func, int jac) {
  Handle* h = (Handle*)vh;
  Solver* s = h->prob->get_solver();
  DofObject* dofs = h->prob->get_dofs();
  const int nf = (int)dofs->n_global_free_dofs(), np = (int)dofs->n_global_const_dofs();
  Vec Up_tmp; VecDuplicate(s->_U.p, &Up_tmp);
  pvector Fext_tmp; VecDuplicate(s->_U.f, &Fext_tmp.f); VecDuplicate(s->_U.p, &Fext_tmp.p);
  h->prob->get_assembler()->assemble_new_load_step(Up_tmp, Fext_tmp, t_frac);
  VecDestroy(&Up_tmp);
  for (int i = 0; i < nf; ++i) s->_U.f->a[i] = U[i];
  for (int i = 0; i < np; ++i) s->_U.p->a[i] = U[nf + i];
  s->store_solution(s->_U, h->prob->get_solution());
  InternalVars* iv = h->prob->get_internal_vars();
  std::vector<std::vector<std::vector<double>>>& all = iv->get_all_internal_vars();
  if (isv_committed) {
    size_t k = 0;
    for (auto& e : all) for (auto& q : e) for (double& v : q) v = isv_committed[k++];
  }
  std::vector<std::vector<std::vector<double>>> trial;
  iv->preallocate_internal_vars_object(trial);
  auto t0 = std::chrono::steady_clock::now();
  h->prob->get_assembler()->assemble(s->_K, s->_P_int, 0.0, trial, h->prob->get_solution(), func != 0, jac != 0);
  auto t1 = std::chrono::steady_clock::now();
  export_mat(h, "K_ff", s->_K.ff);
  export_mat(h, "K_fp", s->_K.fp);
  export_mat(h, "K_pf", s->_K.pf);
  export_mat(h, "K_pp", s->_K.pp);
  export_vec(h, "P_f", s->_P_int.f);
  export_vec(h, "P_p", s->_P_int.p);
  Export& it = put_d(h, "isv_trial");
  for (auto& e : trial) for (auto& q : e) for (double v : q) it.f64.push_back(v);
  // Damage zone of every cohesive quadrature point (Material::get_cohesive_damage_zone on the
  // opening ProblemUtilities::cohesiveDeltaFast forms), in element / cohesive element / qp order.
  Export& zones = put_i(h, "coh_zone");
  Mesh* mesh = h->mesh;
  const id_type nndof = h->prob->get_dofs()->nndof();
  if (mesh->is_cohesive()) {
    for (Mesh::element_iterator eit = mesh->active_elements_begin(); eit != mesh->active_elements_end(); ++eit) {
      Elem* el = *eit;
      if (!el->is_intersected()) continue;
      id_type l_elem = mesh->global_to_local_elem(el->get_id());
      std::vector<double> elem_U;
      ProblemUtilities::formElementalVector(elem_U, el, h->prob->get_solution());
      std::vector<std::vector<short_id_type>>& cs = el->getCohesiveElemStructure();
      id_type curr_qp = mesh->n_volumetric_qps(l_elem);
      for (id_type ce = 0; ce < el->n_cohesive_elem(); ++ce) {
        CohesiveElem* coh_el = el->get_cohesive_elem(ce);
        std::vector<double> cu(coh_el->n_nodes() * nndof);
        for (id_type n = 0; n < coh_el->n_nodes(); ++n)
          for (id_type d = 0; d < nndof; ++d) cu[n * nndof + d] = elem_U[cs[ce][n] * nndof + d];
        Material* mat = el->get_cohesive_material(ce);
        for (id_type q = 0; q < coh_el->n_q_points(); ++q) {
          std::vector<double> delta;
          ProblemUtilities::cohesiveDeltaFast(delta, mesh->get_shape(l_elem, curr_qp), cu, mesh->get_rot_matrix(l_elem, curr_qp));
          zones.i32.push_back((int)mat->get_cohesive_damage_zone(delta));
          curr_qp++;
        }
      }
    }
  }
  return std::chrono::duration<double>(t1 - t0).count();
}

/* Times n_rep calls of Assembler::assemble(K+R) on the state left by pgref_assemble; returns the median seconds. */
/* Problem::homogenize (src/Problem.cpp:471-484) on the state left by the last pgref_assemble;
 * exports "homogenized" (the volume-averaged stress, Voigt). */
void pgref_homogenize(void* vh) {
  Handle* h = (Handle*)vh;
  h->prob->homogenize();
  Export& e = put_d(h, "homogenized");
  e.f64 = h->prob->getHomogenizedValue();
}

/* WriterHomogenization::writeConsecutive (src/WriterHomogenization.cpp:41-61) on the current
 * macroscale value and the last pgref_homogenize result: the reference's homogenization CSV. */
void pgref_write_homogenization(void* vh, const char* filename, double t, int step) {
  Handle* h = (Handle*)vh;
  WriterHomogenization w(h->prob);
  w.writeConsecutive(filename, t, (id_type)step);
}

/* Problem::setMacroscaleValue (include/Problem.h:310): the macroscale strain of a subscale problem;
 * the next pgref_assemble applies it through assemble_new_load_step. */
void pgref_set_macro(void* vh, const double* eps) {
  Handle* h = (Handle*)vh;
  const int n = (h->prob->get_mesh()->dim() == 3) ? 6 : 3;
  std::vector<double> v(eps, eps + n);
  h->prob->setMacroscaleValue(v);
}

double pgref_time_assemble(void* vh, int n_rep) {
  Handle* h = (Handle*)vh;
  Solver* s = h->prob->get_solver();
  InternalVars* iv = h->prob->get_internal_vars();
  std::vector<std::vector<std::vector<double>>> trial;
  iv->preallocate_internal_vars_object(trial);
  std::vector<double> t;
  for (int r = 0; r < n_rep; ++r) {
    auto t0 = std::chrono::steady_clock::now();
    h->prob->get_assembler()->assemble(s->_K, s->_P_int, 0.0, trial, h->prob->get_solution(), true, true);
    auto t1 = std::chrono::steady_clock::now();
    t.push_back(std::chrono::duration<double>(t1 - t0).count());
  }
  std::sort(t.begin(), t.end());
  return t.empty() ? 0.0 : t[t.size() / 2];
}

/*
 * Runs the reference's own solve (Problem::solve_problem -> Solver::solve): for a nonlinear
 * problem the adaptive load stepping of src/SolverNonlinear.cpp:70-328 with Newton steps of
 * src/SolverNonlinearKSP.cpp:55-157.  Exports the final displacement ("U_final", free then
 * constrained), the committed internal variables ("isv_final") and the log text ("log").
 */
int pgref_solve(void* vh) {
  Handle* h = (Handle*)vh;
  writeToScreen = false;
  logFile = h->log_path;
  { std::ofstream clr(h->log_path.c_str(), std::ofstream::trunc); }
  Solver* s = h->prob->get_solver();
  s->solve();
  Export& u = put_d(h, "U_final");
  u.f64 = s->_U.f->a;
  u.f64.insert(u.f64.end(), s->_U.p->a.begin(), s->_U.p->a.end());
  Export& iv = put_d(h, "isv_final");
  for (auto& e : h->prob->get_internal_vars()->get_all_internal_vars()) for (auto& q : e) for (double v : q) iv.f64.push_back(v);
  std::ifstream in(h->log_path.c_str());
  std::stringstream ss; ss << in.rdbuf();
  std::string txt = ss.str();
  Export& lg = put_i(h, "log");
  for (char c : txt) lg.i32.push_back((int)(unsigned char)c);
  return 0;
}

/*
 * Attaches a B200 context to this problem through the drop-in Assembler::assemble
 * (pigfem_b200/drop_in/Assembler_b200.cpp): only in the library variant linked with it
 * (_ref/libpigfem_ref_b200.so), where every later Assembler::assemble -- the reference's own
 * solvers included -- runs on the device.  Returns the pg_dropin_bind status, or -1 in the
 * CPU-only library.
 */
int pgref_bind_gpu(void* vh) {
  Handle* h = (Handle*)vh;
  if (!pg_dropin_bind) return -1;
  const pgref_config& c = h->cfg;
  pg_problem_desc d;
  std::memset(&d, 0, sizeof(d));
  d.elem_type = c.elem_type;
  d.n[0] = c.nx; d.n[1] = c.ny; d.n[2] = c.nz;
  d.lo[0] = c.xmin; d.lo[1] = c.ymin; d.lo[2] = c.zmin;
  d.hi[0] = c.xmax; d.hi[1] = c.ymax; d.hi[2] = c.zmax;
  d.n_incl = c.n_incl; d.incl = c.incl;
  d.E_matrix = c.E_matrix; d.nu_matrix = c.nu_matrix; d.E_fiber = c.E_fiber; d.nu_fiber = c.nu_fiber;
  d.coh_law = c.coh_law;
  for (int i = 0; i < 4; ++i) d.coh[i] = c.coh[i];
  d.plane_strain = c.plane_strain; d.subscale = c.subscale;
  for (int i = 0; i < 6; ++i) d.eps_macro[i] = c.eps_macro[i];
  d.app_strain = c.app_strain;
  d.ply_frac = c.ply_frac;
  for (int i = 0; i < 5; ++i) d.ply[i] = c.ply[i];
  return pg_dropin_bind((void*)h->prob, &d);
}

const char* pgref_gpu_error(void) { return pg_dropin_last_error ? pg_dropin_last_error() : "drop-in not linked"; }

/* Named-array access: returns 1 for int32, 2 for float64, 0 if absent; *n gets the length. */
int pgref_get(void* vh, const char* name, long* n, void** ptr) {
  Handle* h = (Handle*)vh;
  auto it = h->out.find(name);
  if (it == h->out.end()) { *n = 0; *ptr = nullptr; return 0; }
  if (it->second.is_int) { *n = (long)it->second.i32.size(); *ptr = it->second.i32.data(); return 1; }
  *n = (long)it->second.f64.size(); *ptr = it->second.f64.data(); return 2;
}

void pgref_destroy(void* vh) {
  Handle* h = (Handle*)vh;
  std::remove(h->log_path.c_str());
  // The reference's Problem/Mesh destructors are not exercised (Mesh::~Mesh calls PetscFinalize);
  // the handle's exports are released.
  h->out.clear();
  delete h;
}

}  // extern "C"
