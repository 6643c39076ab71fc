/*
 * Assembler_b200.cpp -- the reference's Assembler::assemble on the B200 assembly path.
 *
 * Add this translation unit to the reference's build in place of the definition of
 * Assembler::assemble in src/Assembler.cpp:65-146 (the other members of Assembler stay where they
 * are) and link libpigfem_b200.so.  Assembler::assemble is non-virtual and every solver reaches
 * it statically (SolverNonlinearKSP.cpp:62,70,104; SolverLinear.cpp:66-71; SolverNonlinear.cpp),
 * so the replacement is link-level: the solvers, the load stepping and the Newton iteration are
 * the reference's own, unchanged.  After Problem::init / Problem::setup the driver attaches a
 * device context to the problem with pg_dropin_bind (include/pigfem_b200_dropin.h).
 *
 * One call does what the reference's does, with the same argument meaning:
 *   - the displacement comes from `solution` (NodalData, src/NodalData.cpp:74-104): standard
 *     nodes in local order, then enrichment nodes (ids ENRICH_START + k), nndof values each;
 *   - the committed internal variables are the problem's InternalVars ([elem][qp][var]); on
 *     return `update_ISVs` holds the trial values, as InternalVars::copy_data followed by the
 *     material updates leaves it (src/Assembler.cpp:92);
 *   - the macroscale strain of a subscale problem is the assembler's current value, already
 *     scaled by the load fraction in assemble_new_load_step (src/Assembler.cpp:394-511);
 *   - K.ff / K.fp / K.pf / K.pp get every value of their (reference-identical) patterns and
 *     P_int.f / P_int.p their entries when assembleJac / assembleFunc ask for them.  The first
 *     call on a matrix inserts its rows with MatSetValues (that fixes the nonzero structure);
 *     later calls overwrite the value array in place (MatSeqAIJGetArray).
 * Errors come back as a nonzero PetscErrorCode (the PG_ERR_* status) with the message in
 * pg_dropin_last_error(); nothing exits.
 */
#include "Assembler.h"
#include "InternalVars.h"
#include "Mesh.h"
#include "NodalData.h"
#include "Problem.h"
#include "common.h"

#include "../../include/pigfem_b200_dropin.h"

#include <cstring>
#include <map>
#include <mutex>
#include <set>
#include <string>
#include <vector>

namespace {

struct Binding {
  pg_ctx* ctx = nullptr;
  pg_sizes sz{};
  std::vector<int32_t> rowptr[4], cols[4];
  std::set<Mat> pattern_set;           // matrices whose nonzero structure the first call inserted
  std::vector<double> U, isv, vals[4], pf, pp;
};

std::mutex g_mu;
std::map<const void*, Binding*> g_bound;
std::string g_err;

int fail(int code, const std::string& m) {
  std::lock_guard<std::mutex> lock(g_mu);
  g_err = m;
  return code;
}

// Values of one block into its PETSc matrix: on the first call every row is inserted with its
// full column list; afterwards the value array is overwritten in place.
PetscErrorCode put_block(Binding& b, int blk, Mat M) {
  const std::vector<int32_t>& rp = b.rowptr[blk];
  const std::vector<int32_t>& ci = b.cols[blk];
  const std::vector<double>& v = b.vals[blk];
  const int nrows = (int)rp.size() - 1;
  if (b.pattern_set.count(M) == 0) {
    for (int r = 0; r < nrows; ++r) {
      const int n = rp[r + 1] - rp[r];
      if (n == 0) continue;
      PetscErrorCode ierr = MatSetValues(M, 1, &r, n, ci.data() + rp[r], v.data() + rp[r], INSERT_VALUES);
      if (ierr) return ierr;
    }
    b.pattern_set.insert(M);
  } else if (!ci.empty()) {
    PetscScalar* a = nullptr;
    PetscErrorCode ierr = MatSeqAIJGetArray(M, &a);
    if (ierr) return ierr;
    std::memcpy(a, v.data(), v.size() * sizeof(double));
    ierr = MatSeqAIJRestoreArray(M, &a);
    if (ierr) return ierr;
  }
  return 0;
}

}  // namespace

extern "C" int pg_dropin_bind(void* problem, const pg_problem_desc* desc) {
  if (!problem || !desc) return fail(PG_ERR_INPUT, "pg_dropin_bind: null problem or description");
  Binding* b = new Binding;
  int rc = pg_create(desc, &b->ctx);
  if (rc) {
    std::string m = b->ctx ? pg_last_error(b->ctx) : "pg_create failed";
    pg_destroy(b->ctx);
    delete b;
    return fail(rc, "pg_dropin_bind: " + m);
  }
  pg_get_sizes(b->ctx, &b->sz);
  const int nrows[4] = {b->sz.n_free, b->sz.n_free, b->sz.n_const, b->sz.n_const};
  for (int k = 0; k < 4; ++k) {
    b->rowptr[k].resize((size_t)nrows[k] + 1);
    b->cols[k].resize((size_t)b->sz.nnz[k]);
    b->vals[k].resize((size_t)b->sz.nnz[k]);
    pg_get_pattern(b->ctx, k, b->rowptr[k].data(), b->cols[k].data());
  }
  b->U.resize((size_t)b->sz.n_nodes * b->sz.dim);
  b->isv.resize((size_t)b->sz.n_isv);
  b->pf.resize((size_t)b->sz.n_free);
  b->pp.resize((size_t)b->sz.n_const);
  std::lock_guard<std::mutex> lock(g_mu);
  auto it = g_bound.find(problem);
  if (it != g_bound.end()) {
    pg_destroy(it->second->ctx);
    delete it->second;
  }
  g_bound[problem] = b;
  return PG_OK;
}

extern "C" int pg_dropin_unbind(void* problem) {
  std::lock_guard<std::mutex> lock(g_mu);
  auto it = g_bound.find(problem);
  if (it == g_bound.end()) return PG_OK;
  pg_destroy(it->second->ctx);
  delete it->second;
  g_bound.erase(it);
  return PG_OK;
}

extern "C" const char* pg_dropin_last_error(void) {
  std::lock_guard<std::mutex> lock(g_mu);
  return g_err.c_str();
}

PetscErrorCode Assembler::assemble(pmatrix& K, pvector& P_int, double delta_t,
                                   std::vector<std::vector<std::vector<double> > >& update_ISVs, NodalData* solution,
                                   bool assembleFunc, bool assembleJac) {
  (void)delta_t;   // the bulk and cohesive laws on this path are rate-independent
  if (!assembleFunc && !assembleJac) return 0;
  Binding* b = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    auto it = g_bound.find(_prob);
    if (it != g_bound.end()) b = it->second;
  }
  if (!b) return fail(PG_ERR_STATE, "Assembler::assemble: no B200 context bound to this problem (pg_dropin_bind)");
  Mesh* mesh = _prob->get_mesh();
  const int dim = b->sz.dim;
  const id_type n_std = mesh->n_local_nodes(), n_enr = mesh->n_local_enrich_nodes();
  if ((int)(n_std + n_enr) != b->sz.n_nodes || (int)_prob->nndof() != dim)
    return fail(PG_ERR_INPUT, "Assembler::assemble: the mesh does not match the bound context");
  // displacement, node-major: standard nodes then enrichment nodes
  for (id_type n = 0; n < n_std; ++n)
    for (int d = 0; d < dim; ++d) b->U[(size_t)n * dim + d] = solution->get_value_local(n, d);
  for (id_type k = 0; k < n_enr; ++k)
    for (int d = 0; d < dim; ++d) b->U[(size_t)(n_std + k) * dim + d] = solution->get_value_local(ENRICH_START + k, d);
  // committed internal variables
  std::vector<std::vector<std::vector<double> > >& committed = _prob->get_internal_vars()->get_all_internal_vars();
  size_t k = 0;
  for (auto& e : committed)
    for (auto& q : e)
      for (double v : q) {
        if (k >= b->isv.size()) return fail(PG_ERR_INPUT, "Assembler::assemble: internal-variable layout mismatch");
        b->isv[k++] = v;
      }
  if (k != b->isv.size()) return fail(PG_ERR_INPUT, "Assembler::assemble: internal-variable layout mismatch");
  int rc = pg_set_isv(b->ctx, b->isv.data());
  if (rc) return fail(rc, std::string("Assembler::assemble: ") + pg_last_error(b->ctx));
  if (_prob->subscale()) {
    double eps[6] = {0, 0, 0, 0, 0, 0};
    for (size_t i = 0; i < _currentMacroscopicValue.size() && i < 6; ++i) eps[i] = _currentMacroscopicValue[i];
    rc = pg_set_macro_strain(b->ctx, eps);
    if (rc) return fail(rc, std::string("Assembler::assemble: ") + pg_last_error(b->ctx));
  }
  const int flags = (assembleFunc ? PG_FUNC : 0) | (assembleJac ? PG_JAC : 0);
  rc = pg_assemble(b->ctx, b->U.data(), 1.0, flags, b->vals[0].data(), b->vals[1].data(), b->vals[2].data(),
                   b->vals[3].data(), b->pf.data(), b->pp.data());
  if (rc) return fail(rc, std::string("Assembler::assemble: ") + pg_last_error(b->ctx));
  PetscErrorCode ierr = 0;
  if (assembleJac) {
    Mat mats[4] = {K.ff, K.fp, K.pf, K.pp};
    for (int blk = 0; blk < 4; ++blk) {
      ierr = put_block(*b, blk, mats[blk]);CHKERRQ(ierr);
    }
    for (int blk = 0; blk < 4; ++blk) { ierr = MatAssemblyBegin(mats[blk], MAT_FINAL_ASSEMBLY);CHKERRQ(ierr); }
    for (int blk = 0; blk < 4; ++blk) { ierr = MatAssemblyEnd(mats[blk], MAT_FINAL_ASSEMBLY);CHKERRQ(ierr); }
  }
  if (assembleFunc) {
    PetscScalar* a = nullptr;
    ierr = VecGetArray(P_int.f, &a);CHKERRQ(ierr);
    std::memcpy(a, b->pf.data(), b->pf.size() * sizeof(double));
    ierr = VecRestoreArray(P_int.f, &a);CHKERRQ(ierr);
    ierr = VecGetArray(P_int.p, &a);CHKERRQ(ierr);
    std::memcpy(a, b->pp.data(), b->pp.size() * sizeof(double));
    ierr = VecRestoreArray(P_int.p, &a);CHKERRQ(ierr);
    ierr = VecAssemblyBegin(P_int.f);CHKERRQ(ierr);
    ierr = VecAssemblyBegin(P_int.p);CHKERRQ(ierr);
    ierr = VecAssemblyEnd(P_int.f);CHKERRQ(ierr);
    ierr = VecAssemblyEnd(P_int.p);CHKERRQ(ierr);
  }
  // trial internal variables into the caller's structure (shaped like the committed ones)
  _prob->get_internal_vars()->copy_data(update_ISVs);
  rc = pg_get_isv(b->ctx, 1, b->isv.data());
  if (rc) return fail(rc, "Assembler::assemble: reading the trial internal variables failed");
  k = 0;
  for (auto& e : update_ISVs)
    for (auto& q : e)
      for (double& v : q) v = b->isv[k++];
  return 0;
}
