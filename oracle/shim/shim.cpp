/*
 * shim.cpp -- serial implementations behind oracle/shim/include/pgshim.h.
 *
 * TEST INFRASTRUCTURE ONLY: linked into oracle/_ref (the reference PIGFEM compiled from its
 * own sources) so the reference's assembly can act as the parity oracle and CPU baseline.
 *
 *  - MPI: one rank; reductions and scans copy the input (the single-rank result).
 *  - PETSc: sequential AIJ matrices whose rows are kept sorted; MatSetValue(ADD) does a binary
 *    search in the row and inserts a new slot when the column is absent, so the final pattern is
 *    exactly the set of (row, col) locations the caller touched (explicit zeros included), which
 *    is what PETSc's MatAssemblyEnd(FINAL) leaves after compressing unused preallocation.
 *    KSPSolve (PREONLY + CHOLESKY in the reference) is a direct envelope LDL^T factorisation
 *    after reverse Cuthill-McKee reordering, written for this project.
 *  - GSL: plain-loop CBLAS; Steffensen root finding (Newton iterates + Aitken delta-squared
 *    acceleration, as published by Steffensen / Aitken); Brent's method (Brent 1973, "Algorithms
 *    for Minimization without Derivatives", ch. 4); the multiroot "hybridj" solver is replaced by
 *    full Newton steps on the analytic Jacobian (Powell's hybrid method takes exactly the Newton
 *    step whenever it lies inside the trust region, which holds for the well-conditioned inverse
 *    isoparametric maps solved here; results agree to rounding).
 *  - METIS and everything the serial assembly path never reaches abort when called.
 */
#include "pgshim.h"

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <string>
#include <vector>

static void pg_unreachable(const char* what) {
  std::fprintf(stderr, "oracle shim: %s is not implemented (serial assembly path only)\n", what);
  std::abort();
}

static size_t dt_size(MPI_Datatype dt) {
  switch (dt) {
    case MPI_CHAR: case MPI_UNSIGNED_CHAR: case MPI_C_BOOL: return 1;
    case MPI_INT: case MPI_UNSIGNED: case MPI_FLOAT: return 4;
    case MPI_LONG: case MPI_UNSIGNED_LONG: case MPI_DOUBLE: case MPI_LONG_LONG: return 8;
    default: return 0;
  }
}

extern "C" {

/* ---------------------------------------------------------------- MPI */
int MPI_Init(int*, char***) { return 0; }
int MPI_Initialized(int* f) { *f = 1; return 0; }
int MPI_Finalize(void) { return 0; }
int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return 0; }
int MPI_Barrier(MPI_Comm) { return 0; }
static int copy_buf(const void* s, void* r, int count, MPI_Datatype dt) {
  size_t sz = dt_size(dt);
  if (!sz) pg_unreachable("MPI reduction on a derived datatype");
  if (s != r && count > 0) std::memmove(r, s, sz * (size_t)count);
  return 0;
}
int MPI_Allreduce(const void* s, void* r, int c, MPI_Datatype dt, MPI_Op, MPI_Comm) { return copy_buf(s, r, c, dt); }
int MPI_Reduce(const void* s, void* r, int c, MPI_Datatype dt, MPI_Op, int, MPI_Comm) { return copy_buf(s, r, c, dt); }
int MPI_Scan(const void* s, void* r, int c, MPI_Datatype dt, MPI_Op, MPI_Comm) { return copy_buf(s, r, c, dt); }
int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return 0; }
int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm) { pg_unreachable("MPI_Send"); return 1; }
int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*) { pg_unreachable("MPI_Isend"); return 1; }
int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) { pg_unreachable("MPI_Recv"); return 1; }
int MPI_Probe(int, int, MPI_Comm, MPI_Status*) { pg_unreachable("MPI_Probe"); return 1; }
int MPI_Get_count(const MPI_Status*, MPI_Datatype, int*) { pg_unreachable("MPI_Get_count"); return 1; }
int MPI_Waitall(int count, MPI_Request*, MPI_Status*) { if (count) pg_unreachable("MPI_Waitall"); return 0; }
static int g_next_type = 100;
int MPI_Type_create_struct(int, const int*, const MPI_Aint*, const MPI_Datatype*, MPI_Datatype* t) { *t = g_next_type++; return 0; }
int MPI_Type_commit(MPI_Datatype*) { return 0; }
int MPI_Type_free(MPI_Datatype*) { return 0; }

int METIS_PartMeshDual(idx_t*, idx_t*, idx_t*, idx_t*, idx_t*, idx_t*, idx_t*, idx_t*, real_t*, idx_t*, idx_t*, idx_t*, idx_t*) {
  pg_unreachable("METIS_PartMeshDual");
  return 0;
}

}  // extern "C"

#include "pgshim_objects.h"

extern "C" {

PetscErrorCode PetscInitialize(int*, char***, const char*, const char*) { return 0; }
PetscErrorCode PetscFinalize(void) { return 0; }
PetscErrorCode PetscPrintf(MPI_Comm, const char* fmt, ...) {
  va_list ap; va_start(ap, fmt); std::vfprintf(stdout, fmt, ap); va_end(ap); return 0;
}

PetscErrorCode MatCreate(MPI_Comm, Mat* A) { *A = new pg_Mat; return 0; }
PetscErrorCode MatSetSizes(Mat A, PetscInt m, PetscInt n, PetscInt M, PetscInt N) {
  A->m = (m >= 0) ? m : M; A->n = (n >= 0) ? n : N;
  A->cols.assign(A->m, {}); A->vals.assign(A->m, {});
  return 0;
}
PetscErrorCode MatSetType(Mat A, MatType t) {
  A->dense = (std::strstr(t, "dense") != nullptr);
  if (A->dense) A->dvals.assign((size_t)A->m * A->n, 0.0);
  return 0;
}
PetscErrorCode MatSetFromOptions(Mat) { return 0; }
PetscErrorCode MatSetUp(Mat) { return 0; }
PetscErrorCode MatCreateSeqAIJ(MPI_Comm, PetscInt m, PetscInt n, PetscInt, const PetscInt nnz[], Mat* A) {
  *A = new pg_Mat; (*A)->m = m; (*A)->n = n;
  (*A)->cols.assign(m, {}); (*A)->vals.assign(m, {});
  if (nnz) for (int i = 0; i < m; ++i) { (*A)->cols[i].reserve(nnz[i]); (*A)->vals[i].reserve(nnz[i]); }
  return 0;
}
PetscErrorCode MatCreateSeqDense(MPI_Comm, PetscInt m, PetscInt n, PetscScalar*, Mat* A) {
  *A = new pg_Mat; (*A)->m = m; (*A)->n = n; (*A)->dense = true; (*A)->dvals.assign((size_t)m * n, 0.0); return 0;
}
PetscErrorCode MatCreateDense(MPI_Comm c, PetscInt m, PetscInt n, PetscInt M, PetscInt N, PetscScalar* d, Mat* A) {
  return MatCreateSeqDense(c, m >= 0 ? m : M, n >= 0 ? n : N, d, A);
}
PetscErrorCode MatMPIAIJSetPreallocation(Mat, PetscInt, const PetscInt[], PetscInt, const PetscInt[]) { return 0; }
PetscErrorCode MatSetBlockSize(Mat, PetscInt) { return 0; }
PetscErrorCode MatSetOption(Mat, MatOption, PetscBool) { return 0; }
PetscErrorCode MatSetValue(Mat A, PetscInt i, PetscInt j, PetscScalar v, InsertMode mode) {
  if (i < 0 || j < 0 || i >= A->m || j >= A->n) {
    std::fprintf(stderr, "oracle shim: MatSetValue(%d,%d) outside %dx%d\n", i, j, A->m, A->n);
    return 63;
  }
  if (A->dense) {
    double& d = A->dvals[(size_t)i * A->n + j];
    d = (mode == ADD_VALUES) ? d + v : v;
    return 0;
  }
  std::vector<int>& c = A->cols[i];
  auto it = std::lower_bound(c.begin(), c.end(), j);
  size_t k = (size_t)(it - c.begin());
  if (it == c.end() || *it != j) {
    c.insert(it, j);
    A->vals[i].insert(A->vals[i].begin() + k, 0.0);
  }
  double& d = A->vals[i][k];
  d = (mode == ADD_VALUES) ? d + v : v;
  return 0;
}
PetscErrorCode MatSetValues(Mat A, PetscInt m, const PetscInt im[], PetscInt n, const PetscInt in[], const PetscScalar v[], InsertMode mode) {
  for (int a = 0; a < m; ++a)
    for (int b = 0; b < n; ++b) {
      PetscErrorCode e = MatSetValue(A, im[a], in[b], v[a * n + b], mode);
      if (e) return e;
    }
  return 0;
}
PetscErrorCode MatAssemblyBegin(Mat, MatAssemblyType) { return 0; }
PetscErrorCode MatAssemblyEnd(Mat, MatAssemblyType) { return 0; }
PetscErrorCode MatZeroEntries(Mat A) {
  if (A->dense) { std::fill(A->dvals.begin(), A->dvals.end(), 0.0); return 0; }
  for (auto& r : A->vals) std::fill(r.begin(), r.end(), 0.0);
  return 0;
}
// PETSc's SeqAIJ value array: every stored value, rows in order, columns sorted within a row; the
// caller may overwrite it, and RestoreArray writes it back into the rows.
PetscErrorCode MatSeqAIJGetArray(Mat A, PetscScalar** a) {
  if (A->dense) return 56;
  A->flat.clear();
  for (auto& r : A->vals) A->flat.insert(A->flat.end(), r.begin(), r.end());
  *a = A->flat.data();
  return 0;
}
PetscErrorCode MatSeqAIJRestoreArray(Mat A, PetscScalar** a) {
  if (A->dense) return 56;
  size_t k = 0;
  for (auto& r : A->vals)
    for (double& v : r) v = A->flat[k++];
  A->flat.clear();
  if (a) *a = nullptr;
  return 0;
}
PetscErrorCode MatMult(Mat A, Vec x, Vec y) {
  y->a.assign(A->m, 0.0);
  for (int i = 0; i < A->m; ++i) {
    double s = 0.0;
    if (A->dense) for (int j = 0; j < A->n; ++j) s += A->dvals[(size_t)i * A->n + j] * x->a[j];
    else for (size_t k = 0; k < A->cols[i].size(); ++k) s += A->vals[i][k] * x->a[A->cols[i][k]];
    y->a[i] = s;
  }
  return 0;
}
PetscErrorCode MatMultTranspose(Mat A, Vec x, Vec y) {
  y->a.assign(A->n, 0.0);
  for (int i = 0; i < A->m; ++i) {
    if (A->dense) for (int j = 0; j < A->n; ++j) y->a[j] += A->dvals[(size_t)i * A->n + j] * x->a[i];
    else for (size_t k = 0; k < A->cols[i].size(); ++k) y->a[A->cols[i][k]] += A->vals[i][k] * x->a[i];
  }
  return 0;
}
PetscErrorCode MatGetOwnershipRange(Mat A, PetscInt* lo, PetscInt* hi) { if (lo) *lo = 0; if (hi) *hi = A->m; return 0; }
PetscErrorCode MatGetOwnershipRangeColumn(Mat A, PetscInt* lo, PetscInt* hi) { if (lo) *lo = 0; if (hi) *hi = A->n; return 0; }
PetscErrorCode MatGetOrdering(Mat, MatOrderingType, IS*, IS*) { pg_unreachable("MatGetOrdering"); return 1; }
PetscErrorCode MatGetFactor(Mat, MatSolverPackage, MatFactorType, Mat*) { pg_unreachable("MatGetFactor"); return 1; }
PetscErrorCode MatCholeskyFactorSymbolic(Mat, Mat, IS, const MatFactorInfo*) { pg_unreachable("MatCholeskyFactorSymbolic"); return 1; }
PetscErrorCode MatCholeskyFactorNumeric(Mat, Mat, const MatFactorInfo*) { pg_unreachable("MatCholeskyFactorNumeric"); return 1; }
PetscErrorCode MatMatSolve(Mat, Mat, Mat) { pg_unreachable("MatMatSolve"); return 1; }
PetscErrorCode MatGetColumnVector(Mat, Vec, PetscInt) { pg_unreachable("MatGetColumnVector"); return 1; }
PetscErrorCode MatDestroy(Mat* A) { if (A && *A) { delete *A; *A = nullptr; } return 0; }

PetscErrorCode VecCreateSeq(MPI_Comm, PetscInt n, Vec* v) { *v = new pg_Vec; (*v)->a.assign(n, 0.0); return 0; }
PetscErrorCode VecCreateMPI(MPI_Comm c, PetscInt n, PetscInt N, Vec* v) { return VecCreateSeq(c, n >= 0 ? n : N, v); }
PetscErrorCode VecDuplicate(Vec v, Vec* w) { *w = new pg_Vec; (*w)->a.assign(v->a.size(), 0.0); return 0; }
PetscErrorCode VecSetValue(Vec v, PetscInt i, PetscScalar a, InsertMode mode) {
  if (i < 0 || (size_t)i >= v->a.size()) { std::fprintf(stderr, "oracle shim: VecSetValue(%d) outside %zu\n", i, v->a.size()); return 63; }
  v->a[i] = (mode == ADD_VALUES) ? v->a[i] + a : a;
  return 0;
}
PetscErrorCode VecSetValues(Vec v, PetscInt n, const PetscInt ix[], const PetscScalar y[], InsertMode mode) {
  for (int k = 0; k < n; ++k) { PetscErrorCode e = VecSetValue(v, ix[k], y[k], mode); if (e) return e; }
  return 0;
}
PetscErrorCode VecGetValues(Vec v, PetscInt n, const PetscInt ix[], PetscScalar y[]) { for (int k = 0; k < n; ++k) y[k] = v->a[ix[k]]; return 0; }
PetscErrorCode VecAssemblyBegin(Vec) { return 0; }
PetscErrorCode VecAssemblyEnd(Vec) { return 0; }
PetscErrorCode VecZeroEntries(Vec v) { std::fill(v->a.begin(), v->a.end(), 0.0); return 0; }
PetscErrorCode VecSet(Vec v, PetscScalar a) { std::fill(v->a.begin(), v->a.end(), a); return 0; }
PetscErrorCode VecAXPY(Vec y, PetscScalar a, Vec x) { for (size_t i = 0; i < y->a.size(); ++i) y->a[i] += a * x->a[i]; return 0; }
PetscErrorCode VecCopy(Vec x, Vec y) { y->a = x->a; return 0; }
PetscErrorCode VecScale(Vec x, PetscScalar a) { for (double& d : x->a) d *= a; return 0; }
PetscErrorCode VecDot(Vec x, Vec y, PetscScalar* r) { double s = 0; for (size_t i = 0; i < x->a.size(); ++i) s += x->a[i] * y->a[i]; *r = s; return 0; }
PetscErrorCode VecNorm(Vec x, NormType t, PetscReal* r) {
  double s = 0;
  if (t == NORM_2 || t == NORM_FROBENIUS) { for (double d : x->a) s += d * d; s = std::sqrt(s); }
  else if (t == NORM_1) { for (double d : x->a) s += std::fabs(d); }
  else { for (double d : x->a) s = std::max(s, std::fabs(d)); }
  *r = s; return 0;
}
PetscErrorCode VecGetArray(Vec x, PetscScalar** a) { *a = x->a.data(); return 0; }
PetscErrorCode VecRestoreArray(Vec, PetscScalar**) { return 0; }
PetscErrorCode VecGetArrayRead(Vec x, const PetscScalar** a) { *a = x->a.data(); return 0; }
PetscErrorCode VecRestoreArrayRead(Vec, const PetscScalar**) { return 0; }
PetscErrorCode VecGetOwnershipRange(Vec x, PetscInt* lo, PetscInt* hi) { if (lo) *lo = 0; if (hi) *hi = (PetscInt)x->a.size(); return 0; }
PetscErrorCode VecGetSize(Vec x, PetscInt* n) { *n = (PetscInt)x->a.size(); return 0; }
PetscErrorCode VecGetLocalSize(Vec x, PetscInt* n) { *n = (PetscInt)x->a.size(); return 0; }
PetscErrorCode VecDestroy(Vec* v) { if (v && *v) { delete *v; *v = nullptr; } return 0; }
PetscErrorCode VecScatterCreate(Vec, IS, Vec, IS, VecScatter*) { pg_unreachable("VecScatterCreate"); return 1; }
PetscErrorCode VecScatterCreateToAll(Vec, VecScatter*, Vec*) { pg_unreachable("VecScatterCreateToAll"); return 1; }
PetscErrorCode VecScatterBegin(VecScatter, Vec, Vec, InsertMode, ScatterMode) { pg_unreachable("VecScatterBegin"); return 1; }
PetscErrorCode VecScatterEnd(VecScatter, Vec, Vec, InsertMode, ScatterMode) { pg_unreachable("VecScatterEnd"); return 1; }
PetscErrorCode VecScatterDestroy(VecScatter* s) { if (s) *s = nullptr; return 0; }

PetscErrorCode ISCreateGeneral(MPI_Comm, PetscInt n, const PetscInt idx[], PetscCopyMode, IS* is) {
  *is = new pg_IS; (*is)->idx.assign(idx, idx + n); return 0;
}
PetscErrorCode ISDestroy(IS* is) { if (is && *is) { delete *is; *is = nullptr; } return 0; }

/* ---------------------------------------------------------------- direct solver for KSPSolve */
// Envelope (skyline) LDL^T of the symmetric matrix A after a reverse Cuthill-McKee permutation.
static int envelope_ldlt_solve(const pg_Mat& A, const std::vector<double>& b, std::vector<double>& x) {
  const int n = A.m;
  x.assign(n, 0.0);
  if (n == 0) return 0;
  // symmetric adjacency
  std::vector<std::vector<int>> adj(n);
  for (int i = 0; i < n; ++i)
    for (int j : A.cols[i]) if (j != i) { adj[i].push_back(j); adj[j].push_back(i); }
  for (auto& a : adj) { std::sort(a.begin(), a.end()); a.erase(std::unique(a.begin(), a.end()), a.end()); }
  // RCM ordering, component by component, each started from a minimum-degree vertex
  std::vector<int> order; order.reserve(n);
  std::vector<char> seen(n, 0);
  std::vector<int> by_degree(n);
  for (int i = 0; i < n; ++i) by_degree[i] = i;
  std::stable_sort(by_degree.begin(), by_degree.end(), [&](int a, int b) { return adj[a].size() < adj[b].size(); });
  for (int s : by_degree) {
    if (seen[s]) continue;
    std::deque<int> q; q.push_back(s); seen[s] = 1;
    while (!q.empty()) {
      int v = q.front(); q.pop_front(); order.push_back(v);
      std::vector<int> nb;
      for (int w : adj[v]) if (!seen[w]) { seen[w] = 1; nb.push_back(w); }
      std::stable_sort(nb.begin(), nb.end(), [&](int a, int b) { return adj[a].size() < adj[b].size(); });
      for (int w : nb) q.push_back(w);
    }
  }
  std::reverse(order.begin(), order.end());
  std::vector<int> pos(n);
  for (int k = 0; k < n; ++k) pos[order[k]] = k;
  // envelope: first[k] = smallest permuted column in row k (lower triangle)
  std::vector<int> first(n);
  for (int k = 0; k < n; ++k) {
    int f = k;
    for (int w : adj[order[k]]) f = std::min(f, pos[w]);
    first[k] = f;
  }
  std::vector<size_t> start(n + 1, 0);
  for (int k = 0; k < n; ++k) start[k + 1] = start[k] + (size_t)(k - first[k] + 1);
  std::vector<double> L(start[n], 0.0);  // row k holds columns first[k]..k
  for (int i = 0; i < n; ++i) {
    int ki = pos[i];
    for (size_t t = 0; t < A.cols[i].size(); ++t) {
      int kj = pos[A.cols[i][t]];
      if (kj <= ki) L[start[ki] + (size_t)(kj - first[ki])] = A.vals[i][t];
    }
  }
  std::vector<double> D(n, 0.0);
  for (int k = 0; k < n; ++k) {
    double* Lk = &L[start[k]];
    const int fk = first[k];
    // L(k,j) for j < k:  (A(k,j) - sum_{m<j} L(k,m) D(m) L(j,m)) / D(j)
    for (int j = fk; j < k; ++j) {
      const double* Lj = &L[start[j]];
      const int fj = first[j];
      int m0 = std::max(fk, fj);
      double s = Lk[j - fk];
      for (int m = m0; m < j; ++m) s -= Lk[m - fk] * D[m] * Lj[m - fj];
      Lk[j - fk] = s / D[j];
    }
    double d = Lk[k - fk];
    for (int m = fk; m < k; ++m) d -= Lk[m - fk] * Lk[m - fk] * D[m];
    if (d == 0.0 || !std::isfinite(d)) return 71;
    D[k] = d;
    Lk[k - fk] = 1.0;
  }
  std::vector<double> y(n);
  for (int k = 0; k < n; ++k) y[k] = b[order[k]];
  for (int k = 0; k < n; ++k) {
    const double* Lk = &L[start[k]];
    double s = y[k];
    for (int m = first[k]; m < k; ++m) s -= Lk[m - first[k]] * y[m];
    y[k] = s;
  }
  for (int k = 0; k < n; ++k) y[k] /= D[k];
  for (int k = n - 1; k >= 0; --k) {
    const double* Lk = &L[start[k]];
    for (int m = first[k]; m < k; ++m) y[m] -= Lk[m - first[k]] * y[k];
  }
  for (int k = 0; k < n; ++k) x[order[k]] = y[k];
  return 0;
}

PetscErrorCode KSPCreate(MPI_Comm, KSP* k) { *k = new pg_KSP; return 0; }
PetscErrorCode KSPSetOperators(KSP k, Mat A, Mat) { k->A = A; return 0; }
PetscErrorCode KSPGetPC(KSP k, PC* pc) { *pc = &k->pc; return 0; }
PetscErrorCode KSPSetType(KSP k, KSPType t) { k->type = t; return 0; }
PetscErrorCode KSPCGSetType(KSP, KSPCGType) { return 0; }
PetscErrorCode KSPSetTolerances(KSP, PetscReal, PetscReal, PetscReal, PetscInt) { return 0; }
PetscErrorCode KSPSetFromOptions(KSP) { return 0; }
PetscErrorCode KSPSetUp(KSP) { return 0; }
PetscErrorCode KSPSolve(KSP k, Vec b, Vec x) {
  if (!k->A || k->A->dense) pg_unreachable("KSPSolve without a sparse operator");
  std::vector<double> sol;
  int e = envelope_ldlt_solve(*k->A, b->a, sol);
  if (e) { std::fprintf(stderr, "oracle shim: KSPSolve hit a zero or non-finite pivot\n"); return e; }
  x->a = sol;
  return 0;
}
PetscErrorCode KSPSolveTranspose(KSP k, Vec b, Vec x) { return KSPSolve(k, b, x); }
PetscErrorCode KSPGetIterationNumber(KSP, PetscInt* its) { *its = 1; return 0; }
PetscErrorCode KSPDestroy(KSP* k) { if (k && *k) { delete *k; *k = nullptr; } return 0; }
PetscErrorCode PCSetType(PC pc, PCType t) { pc->type = t; return 0; }
PetscErrorCode PCFactorSetMatSolverPackage(PC, MatSolverPackage) { return 0; }
PetscErrorCode PCSetCoordinates(PC, PetscInt, PetscInt, PetscReal*) { return 0; }
PetscErrorCode PCHYPRESetType(PC, const char*) { return 0; }

PetscErrorCode SNESCreate(MPI_Comm, SNES*) { pg_unreachable("SNESCreate"); return 1; }
PetscErrorCode SNESSetType(SNES, SNESType) { pg_unreachable("SNESSetType"); return 1; }
PetscErrorCode SNESSetFunction(SNES, Vec, PetscErrorCode (*)(SNES, Vec, Vec, void*), void*) { pg_unreachable("SNES"); return 1; }
PetscErrorCode SNESSetJacobian(SNES, Mat, Mat, PetscErrorCode (*)(SNES, Vec, Mat, Mat, void*), void*) { pg_unreachable("SNES"); return 1; }
PetscErrorCode SNESMonitorSet(SNES, PetscErrorCode (*)(SNES, PetscInt, PetscReal, void*), void*, PetscErrorCode (*)(void**)) { pg_unreachable("SNES"); return 1; }
PetscErrorCode SNESSetTolerances(SNES, PetscReal, PetscReal, PetscReal, PetscInt, PetscInt) { pg_unreachable("SNES"); return 1; }
PetscErrorCode SNESGetKSP(SNES, KSP*) { pg_unreachable("SNES"); return 1; }
PetscErrorCode SNESSetFromOptions(SNES) { pg_unreachable("SNES"); return 1; }
PetscErrorCode SNESSolve(SNES, Vec, Vec) { pg_unreachable("SNES"); return 1; }
PetscErrorCode SNESGetFunctionNorm(SNES, PetscReal*) { pg_unreachable("SNES"); return 1; }
PetscErrorCode SNESGetConvergedReason(SNES, SNESConvergedReason*) { pg_unreachable("SNES"); return 1; }
PetscErrorCode SNESDestroy(SNES* s) { if (s) *s = nullptr; return 0; }

/* ---------------------------------------------------------------- GSL vectors / matrices */
gsl_vector* gsl_vector_alloc(size_t n) {
  gsl_vector* v = (gsl_vector*)std::calloc(1, sizeof(gsl_vector));
  v->size = n; v->stride = 1; v->data = (double*)std::calloc(n ? n : 1, sizeof(double)); v->owner = 1;
  return v;
}
gsl_vector* gsl_vector_calloc(size_t n) { return gsl_vector_alloc(n); }
void gsl_vector_free(gsl_vector* v) { if (!v) return; if (v->owner) std::free(v->data); std::free(v); }
double gsl_vector_get(const gsl_vector* v, size_t i) { return v->data[i * v->stride]; }
void gsl_vector_set(gsl_vector* v, size_t i, double x) { v->data[i * v->stride] = x; }
gsl_matrix* gsl_matrix_alloc(size_t n1, size_t n2) {
  gsl_matrix* m = (gsl_matrix*)std::calloc(1, sizeof(gsl_matrix));
  m->size1 = n1; m->size2 = n2; m->tda = n2; m->data = (double*)std::calloc(n1 * n2 ? n1 * n2 : 1, sizeof(double)); m->owner = 1;
  return m;
}
void gsl_matrix_free(gsl_matrix* m) { if (!m) return; if (m->owner) std::free(m->data); std::free(m); }
double gsl_matrix_get(const gsl_matrix* m, size_t i, size_t j) { return m->data[i * m->tda + j]; }
void gsl_matrix_set(gsl_matrix* m, size_t i, size_t j, double x) { m->data[i * m->tda + j] = x; }
gsl_matrix_view gsl_matrix_view_array(double* base, size_t n1, size_t n2) {
  gsl_matrix_view v; v.matrix.size1 = n1; v.matrix.size2 = n2; v.matrix.tda = n2; v.matrix.data = base; v.matrix.block = nullptr; v.matrix.owner = 0;
  return v;
}

/* ---------------------------------------------------------------- GSL 1-D root finding */
struct pg_root_fdfsolver {
  const gsl_root_fdfsolver_type* type;
  gsl_function_fdf* fdf;
  double root;
  double x, x_1, x_2, f, df;
  int count;
};
struct pg_root_fsolver {
  const gsl_root_fsolver_type* type;
  gsl_function* F;
  double root, x_lower, x_upper;
  // Brent state: a, b, c bracket points and their function values, step sizes d, e
  double a, b, c, d, e, fa, fb, fc;
};
static const gsl_root_fdfsolver_type k_steff = {"steffenson"};
static const gsl_root_fdfsolver_type k_newton = {"newton"};
static const gsl_root_fsolver_type k_brent = {"brent"};
static const gsl_root_fsolver_type k_bisect = {"bisection"};
const gsl_root_fdfsolver_type* gsl_root_fdfsolver_steffenson = &k_steff;
const gsl_root_fdfsolver_type* gsl_root_fdfsolver_newton = &k_newton;
const gsl_root_fsolver_type* gsl_root_fsolver_brent = &k_brent;
const gsl_root_fsolver_type* gsl_root_fsolver_bisection = &k_bisect;

gsl_root_fdfsolver* gsl_root_fdfsolver_alloc(const gsl_root_fdfsolver_type* T) {
  gsl_root_fdfsolver* s = new gsl_root_fdfsolver(); s->type = T; return s;
}
int gsl_root_fdfsolver_set(gsl_root_fdfsolver* s, gsl_function_fdf* fdf, double root) {
  s->fdf = fdf; s->root = root; s->x = root; s->x_1 = 0; s->x_2 = 0; s->count = 1;
  fdf->fdf(root, fdf->params, &s->f, &s->df);
  return GSL_SUCCESS;
}
// One Newton step from the current iterate; once three Newton iterates exist, the reported
// root is their Aitken delta-squared extrapolation (Steffensen acceleration).
int gsl_root_fdfsolver_iterate(gsl_root_fdfsolver* s) {
  if (s->df == 0.0) return GSL_EZERODIV;
  double x_new = s->x - s->f / s->df;
  double f_new, df_new;
  s->fdf->fdf(x_new, s->fdf->params, &f_new, &df_new);
  s->x_2 = s->x_1; s->x_1 = s->x; s->x = x_new; s->f = f_new; s->df = df_new;
  if (!std::isfinite(f_new)) return GSL_EBADFUNC;
  if (s->type == &k_steff && s->count >= 3) {
    double u = s->x_1 - s->x_2;
    double v = s->x - 2.0 * s->x_1 + s->x_2;
    s->root = (v == 0.0) ? s->x : s->x_2 - u * u / v;
  } else {
    s->root = s->x;
    s->count++;
  }
  return GSL_SUCCESS;
}
double gsl_root_fdfsolver_root(const gsl_root_fdfsolver* s) { return s->root; }
void gsl_root_fdfsolver_free(gsl_root_fdfsolver* s) { delete s; }

gsl_root_fsolver* gsl_root_fsolver_alloc(const gsl_root_fsolver_type* T) { gsl_root_fsolver* s = new gsl_root_fsolver(); s->type = T; return s; }
int gsl_root_fsolver_set(gsl_root_fsolver* s, gsl_function* F, double lo, double hi) {
  s->F = F; s->x_lower = lo; s->x_upper = hi; s->root = 0.5 * (lo + hi);
  s->a = lo; s->b = hi; s->fa = F->function(lo, F->params); s->fb = F->function(hi, F->params);
  s->c = s->a; s->fc = s->fa; s->d = s->b - s->a; s->e = s->d;
  if ((s->fa < 0 && s->fb < 0) || (s->fa > 0 && s->fb > 0)) return GSL_EDOM;
  return GSL_SUCCESS;
}
// Brent's method: keep a bracket [b, c] with f(b) f(c) <= 0, b the best estimate; try inverse
// quadratic interpolation (or the secant step when only two distinct points exist), fall back to
// bisection whenever the interpolated step is not safely inside the bracket or not shrinking fast.
int gsl_root_fsolver_iterate(gsl_root_fsolver* s) {
  if (s->type == &k_bisect) {
    double m = 0.5 * (s->x_lower + s->x_upper);
    double fm = s->F->function(m, s->F->params);
    double flo = s->F->function(s->x_lower, s->F->params);
    if ((fm < 0) == (flo < 0)) s->x_lower = m; else s->x_upper = m;
    s->root = 0.5 * (s->x_lower + s->x_upper);
    return GSL_SUCCESS;
  }
  double a = s->a, b = s->b, c = s->c, fa = s->fa, fb = s->fb, fc = s->fc, d = s->d, e = s->e;
  if ((fb < 0 && fc < 0) || (fb > 0 && fc > 0)) { c = a; fc = fa; d = b - a; e = d; }
  if (std::fabs(fc) < std::fabs(fb)) { a = b; b = c; c = a; fa = fb; fb = fc; fc = fa; }
  const double tol = 0.5 * 2.220446049250313e-16 * std::fabs(b);
  const double m = 0.5 * (c - b);
  if (fb == 0.0) {
    s->root = b; s->x_lower = b; s->x_upper = b;
    s->a = a; s->b = b; s->c = c; s->fa = fa; s->fb = fb; s->fc = fc; s->d = d; s->e = e;
    return GSL_SUCCESS;
  }
  if (std::fabs(m) <= tol) {
    s->root = b;
    if (b < c) { s->x_lower = b; s->x_upper = c; } else { s->x_lower = c; s->x_upper = b; }
    s->a = a; s->b = b; s->c = c; s->fa = fa; s->fb = fb; s->fc = fc; s->d = d; s->e = e;
    return GSL_SUCCESS;
  }
  if (std::fabs(e) < tol || std::fabs(fa) <= std::fabs(fb)) {
    d = m; e = m;
  } else {
    double p, q, r, ss = fb / fa;
    if (a == c) { p = 2 * m * ss; q = 1 - ss; }
    else {
      q = fa / fc; r = fb / fc;
      p = ss * (2 * m * q * (q - r) - (b - a) * (r - 1));
      q = (q - 1) * (r - 1) * (ss - 1);
    }
    if (p > 0) q = -q; else p = -p;
    if (2 * p < std::min(3 * m * q - std::fabs(tol * q), std::fabs(e * q))) { e = d; d = p / q; }
    else { d = m; e = m; }
  }
  a = b; fa = fb;
  if (std::fabs(d) > tol) b += d; else b += (m > 0 ? +tol : -tol);
  fb = s->F->function(b, s->F->params);
  if (!std::isfinite(fb)) return GSL_EBADFUNC;
  s->root = b;
  if ((fb < 0 && fc < 0) || (fb > 0 && fc > 0)) c = a;
  if (b < c) { s->x_lower = b; s->x_upper = c; } else { s->x_lower = c; s->x_upper = b; }
  s->a = a; s->b = b; s->c = c; s->fa = fa; s->fb = fb; s->fc = (c == a) ? fa : fc; s->d = d; s->e = e;
  return GSL_SUCCESS;
}
double gsl_root_fsolver_root(const gsl_root_fsolver* s) { return s->root; }
double gsl_root_fsolver_x_lower(const gsl_root_fsolver* s) { return s->x_lower; }
double gsl_root_fsolver_x_upper(const gsl_root_fsolver* s) { return s->x_upper; }
void gsl_root_fsolver_free(gsl_root_fsolver* s) { delete s; }

// Converged when |x1 - x0| < epsabs + epsrel * min(|x1|, |x0|) (documented GSL test).
int gsl_root_test_delta(double x1, double x0, double epsabs, double epsrel) {
  const double tol = epsabs + epsrel * std::min(std::fabs(x1), std::fabs(x0));
  if (x1 == x0) return GSL_SUCCESS;
  return (std::fabs(x1 - x0) < tol) ? GSL_SUCCESS : GSL_CONTINUE;
}
int gsl_root_test_interval(double lo, double hi, double epsabs, double epsrel) {
  double min_abs = (lo > 0 && hi > 0) || (lo < 0 && hi < 0) ? std::min(std::fabs(lo), std::fabs(hi)) : 0.0;
  return (std::fabs(hi - lo) < epsabs + epsrel * min_abs) ? GSL_SUCCESS : GSL_CONTINUE;
}

/* ---------------------------------------------------------------- GSL multiroot (Newton steps) */
static const gsl_multiroot_fdfsolver_type k_hybridj = {"hybridj"};
static const gsl_multiroot_fdfsolver_type k_hybridsj = {"hybridsj"};
static const gsl_multiroot_fdfsolver_type k_mnewton = {"newton"};
const gsl_multiroot_fdfsolver_type* gsl_multiroot_fdfsolver_hybridj = &k_hybridj;
const gsl_multiroot_fdfsolver_type* gsl_multiroot_fdfsolver_hybridsj = &k_hybridsj;
const gsl_multiroot_fdfsolver_type* gsl_multiroot_fdfsolver_newton = &k_mnewton;

gsl_multiroot_fdfsolver* gsl_multiroot_fdfsolver_alloc(const gsl_multiroot_fdfsolver_type* T, size_t n) {
  gsl_multiroot_fdfsolver* s = (gsl_multiroot_fdfsolver*)std::calloc(1, sizeof(gsl_multiroot_fdfsolver));
  s->type = T; s->x = gsl_vector_alloc(n); s->f = gsl_vector_alloc(n); s->dx = gsl_vector_alloc(n); s->J = gsl_matrix_alloc(n, n);
  return s;
}
int gsl_multiroot_fdfsolver_set(gsl_multiroot_fdfsolver* s, gsl_multiroot_function_fdf* fdf, const gsl_vector* x) {
  s->fdf = fdf;
  for (size_t i = 0; i < x->size; ++i) gsl_vector_set(s->x, i, gsl_vector_get(x, i));
  return fdf->fdf(s->x, fdf->params, s->f, s->J);
}
// Solve J dx = -f by Gaussian elimination with partial pivoting, x += dx, re-evaluate.
int gsl_multiroot_fdfsolver_iterate(gsl_multiroot_fdfsolver* s) {
  const size_t n = s->x->size;
  std::vector<double> M(n * n), r(n);
  for (size_t i = 0; i < n; ++i) { r[i] = -gsl_vector_get(s->f, i); for (size_t j = 0; j < n; ++j) M[i * n + j] = gsl_matrix_get(s->J, i, j); }
  for (size_t k = 0; k < n; ++k) {
    size_t p = k;
    for (size_t i = k + 1; i < n; ++i) if (std::fabs(M[i * n + k]) > std::fabs(M[p * n + k])) p = i;
    if (M[p * n + k] == 0.0) return GSL_ENOPROGJ;
    if (p != k) { for (size_t j = 0; j < n; ++j) std::swap(M[p * n + j], M[k * n + j]); std::swap(r[p], r[k]); }
    for (size_t i = k + 1; i < n; ++i) {
      double l = M[i * n + k] / M[k * n + k];
      for (size_t j = k; j < n; ++j) M[i * n + j] -= l * M[k * n + j];
      r[i] -= l * r[k];
    }
  }
  for (size_t k = n; k-- > 0;) {
    double t = r[k];
    for (size_t j = k + 1; j < n; ++j) t -= M[k * n + j] * r[j];
    r[k] = t / M[k * n + k];
  }
  for (size_t i = 0; i < n; ++i) { gsl_vector_set(s->dx, i, r[i]); gsl_vector_set(s->x, i, gsl_vector_get(s->x, i) + r[i]); }
  return s->fdf->fdf(s->x, s->fdf->params, s->f, s->J);
}
void gsl_multiroot_fdfsolver_free(gsl_multiroot_fdfsolver* s) {
  if (!s) return; gsl_vector_free(s->x); gsl_vector_free(s->f); gsl_vector_free(s->dx); gsl_matrix_free(s->J); std::free(s);
}
int gsl_multiroot_test_residual(const gsl_vector* f, double epsabs) {
  double sum = 0.0;
  for (size_t i = 0; i < f->size; ++i) sum += std::fabs(gsl_vector_get(f, i));
  return (sum < epsabs) ? GSL_SUCCESS : GSL_CONTINUE;
}

gsl_eigen_symm_workspace* gsl_eigen_symm_alloc(size_t) { pg_unreachable("gsl_eigen_symm_alloc"); return nullptr; }
int gsl_eigen_symm(gsl_matrix*, gsl_vector*, gsl_eigen_symm_workspace*) { pg_unreachable("gsl_eigen_symm"); return 1; }
void gsl_eigen_symm_free(gsl_eigen_symm_workspace*) {}

/* ---------------------------------------------------------------- CBLAS (plain loops) */
void cblas_daxpy(const int N, const double alpha, const double* X, const int incX, double* Y, const int incY) {
  for (int i = 0; i < N; ++i) Y[i * incY] += alpha * X[i * incX];
}
void cblas_saxpy(const int N, const float alpha, const float* X, const int incX, float* Y, const int incY) {
  for (int i = 0; i < N; ++i) Y[i * incY] += alpha * X[i * incX];
}
void cblas_dscal(const int N, const double alpha, double* X, const int incX) { for (int i = 0; i < N; ++i) X[i * incX] *= alpha; }
void cblas_sscal(const int N, const float alpha, float* X, const int incX) { for (int i = 0; i < N; ++i) X[i * incX] *= alpha; }
double cblas_ddot(const int N, const double* X, const int incX, const double* Y, const int incY) {
  double s = 0.0; for (int i = 0; i < N; ++i) s += X[i * incX] * Y[i * incY]; return s;
}
}  // extern "C"

template <typename T>
static void gemv_impl(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE tr, int M, int N, T alpha, const T* A, int lda,
                      const T* X, int incX, T beta, T* Y, int incY) {
  if (order != CblasRowMajor) pg_unreachable("column-major gemv");
  if (tr == CblasNoTrans) {
    for (int i = 0; i < M; ++i) {
      T s = 0; for (int j = 0; j < N; ++j) s += A[i * lda + j] * X[j * incX];
      Y[i * incY] = alpha * s + (beta == T(0) ? T(0) : beta * Y[i * incY]);
    }
  } else {
    for (int j = 0; j < N; ++j) Y[j * incY] = (beta == T(0) ? T(0) : beta * Y[j * incY]);
    for (int i = 0; i < M; ++i) {
      T xi = alpha * X[i * incX];
      for (int j = 0; j < N; ++j) Y[j * incY] += A[i * lda + j] * xi;
    }
  }
}
template <typename T>
static void gemm_impl(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE ta, enum CBLAS_TRANSPOSE tb, int M, int N, int K,
                      T alpha, const T* A, int lda, const T* B, int ldb, T beta, T* C, int ldc) {
  if (order != CblasRowMajor) pg_unreachable("column-major gemm");
  for (int i = 0; i < M; ++i)
    for (int j = 0; j < N; ++j) {
      T s = 0;
      for (int k = 0; k < K; ++k) {
        T a = (ta == CblasNoTrans) ? A[i * lda + k] : A[k * lda + i];
        T b = (tb == CblasNoTrans) ? B[k * ldb + j] : B[j * ldb + k];
        s += a * b;
      }
      C[i * ldc + j] = alpha * s + (beta == T(0) ? T(0) : beta * C[i * ldc + j]);
    }
}
extern "C" {
void cblas_dgemv(const enum CBLAS_ORDER o, const enum CBLAS_TRANSPOSE t, const int M, const int N, const double alpha, const double* A,
                 const int lda, const double* X, const int incX, const double beta, double* Y, const int incY) {
  gemv_impl<double>(o, t, M, N, alpha, A, lda, X, incX, beta, Y, incY);
}
void cblas_sgemv(const enum CBLAS_ORDER o, const enum CBLAS_TRANSPOSE t, const int M, const int N, const float alpha, const float* A,
                 const int lda, const float* X, const int incX, const float beta, float* Y, const int incY) {
  gemv_impl<float>(o, t, M, N, alpha, A, lda, X, incX, beta, Y, incY);
}
void cblas_dgemm(const enum CBLAS_ORDER o, const enum CBLAS_TRANSPOSE ta, const enum CBLAS_TRANSPOSE tb, const int M, const int N,
                 const int K, const double alpha, const double* A, const int lda, const double* B, const int ldb, const double beta,
                 double* C, const int ldc) {
  gemm_impl<double>(o, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
}
void cblas_sgemm(const enum CBLAS_ORDER o, const enum CBLAS_TRANSPOSE ta, const enum CBLAS_TRANSPOSE tb, const int M, const int N,
                 const int K, const float alpha, const float* A, const int lda, const float* B, const int ldb, const float beta,
                 float* C, const int ldc) {
  gemm_impl<float>(o, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
}

}  // extern "C"
