/*
 * pgshim.h -- single-process stand-ins for the PETSc 3.7, MPI, GSL 2.1 and METIS 5.1
 * interfaces that the reference PIGFEM sources include.
 *
 * TEST INFRASTRUCTURE ONLY.  This header lets the oracle build compile the reference's own
 * C++ sources (unmodified, where they lie) on a machine that has none of those libraries,
 * so that the reference's assembly can be run as the parity oracle.  Only the serial subset
 * that the assembly path executes is implemented (oracle/shim/shim.cpp); every other entry
 * point aborts loudly if it is ever reached.
 *
 * Declarations follow the public API documentation of each library (names, argument order,
 * argument meaning).  No library source is reproduced.
 */
#pragma once

#include <stddef.h>
#include <math.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ MPI (one rank) */
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef long MPI_Aint;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; int count_bytes; } MPI_Status;

#define MPI_COMM_WORLD 1
#define MPI_COMM_SELF 2
#define MPI_SUCCESS 0
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_REQUEST_NULL 0

#define MPI_CHAR 1
#define MPI_UNSIGNED_CHAR 2
#define MPI_INT 3
#define MPI_UNSIGNED 4
#define MPI_LONG 5
#define MPI_UNSIGNED_LONG 6
#define MPI_FLOAT 7
#define MPI_DOUBLE 8
#define MPI_C_BOOL 9
#define MPI_LONG_LONG 10

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_LOR 4
#define MPI_LAND 5

int MPI_Init(int* argc, char*** argv);
int MPI_Initialized(int* flag);
int MPI_Finalize(void);
int MPI_Comm_rank(MPI_Comm comm, int* rank);
int MPI_Comm_size(MPI_Comm comm, int* size);
int MPI_Barrier(MPI_Comm comm);
int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype dt, MPI_Op op, MPI_Comm comm);
int MPI_Reduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype dt, MPI_Op op, int root, MPI_Comm comm);
int MPI_Scan(const void* sendbuf, void* recvbuf, int count, MPI_Datatype dt, MPI_Op op, MPI_Comm comm);
int MPI_Bcast(void* buf, int count, MPI_Datatype dt, int root, MPI_Comm comm);
int MPI_Send(const void* buf, int count, MPI_Datatype dt, int dest, int tag, MPI_Comm comm);
int MPI_Isend(const void* buf, int count, MPI_Datatype dt, int dest, int tag, MPI_Comm comm, MPI_Request* req);
int MPI_Recv(void* buf, int count, MPI_Datatype dt, int source, int tag, MPI_Comm comm, MPI_Status* st);
int MPI_Probe(int source, int tag, MPI_Comm comm, MPI_Status* st);
int MPI_Get_count(const MPI_Status* st, MPI_Datatype dt, int* count);
int MPI_Waitall(int count, MPI_Request* reqs, MPI_Status* sts);
int MPI_Type_create_struct(int count, const int* blocklens, const MPI_Aint* displs, const MPI_Datatype* types, MPI_Datatype* newtype);
int MPI_Type_commit(MPI_Datatype* dt);
int MPI_Type_free(MPI_Datatype* dt);

/* ------------------------------------------------------------------ METIS */
typedef int idx_t;
typedef float real_t;
#define METIS_OK 1
int METIS_PartMeshDual(idx_t* ne, idx_t* nn, idx_t* eptr, idx_t* eind, idx_t* vwgt, idx_t* vsize,
                       idx_t* ncommon, idx_t* nparts, real_t* tpwgts, idx_t* options, idx_t* objval,
                       idx_t* epart, idx_t* npart);

/* ------------------------------------------------------------------ PETSc (sequential) */
typedef int PetscErrorCode;
typedef int PetscInt;
typedef double PetscScalar;
typedef double PetscReal;
typedef enum { PETSC_FALSE = 0, PETSC_TRUE = 1 } PetscBool;
typedef struct pg_Mat* Mat;
typedef struct pg_Vec* Vec;
typedef struct pg_KSP* KSP;
typedef struct pg_PC* PC;
typedef struct pg_IS* IS;
typedef struct pg_SNES* SNES;
typedef struct pg_VecScatter* VecScatter;
typedef const char* MatType;
typedef const char* KSPType;
typedef const char* PCType;
typedef const char* SNESType;
typedef const char* MatSolverPackage;
typedef const char* MatOrderingType;
typedef struct { double fill, levels, dtcol, zeropivot, pivotinblocks, shifttype, shiftamount; } MatFactorInfo;
typedef enum { INSERT_VALUES = 1, ADD_VALUES = 2 } InsertMode;
typedef enum { MAT_FLUSH_ASSEMBLY = 1, MAT_FINAL_ASSEMBLY = 0 } MatAssemblyType;
typedef enum { NORM_1 = 0, NORM_2 = 1, NORM_FROBENIUS = 2, NORM_INFINITY = 3 } NormType;
typedef enum { SCATTER_FORWARD = 0, SCATTER_REVERSE = 1 } ScatterMode;
typedef enum { KSP_CG_SYMMETRIC = 0, KSP_CG_HERMITIAN = 1 } KSPCGType;
typedef enum { MAT_FACTOR_NONE, MAT_FACTOR_LU, MAT_FACTOR_CHOLESKY, MAT_FACTOR_ILU, MAT_FACTOR_ICC } MatFactorType;
typedef enum { PETSC_COPY_VALUES, PETSC_OWN_POINTER, PETSC_USE_POINTER } PetscCopyMode;
typedef enum {
  MAT_ROW_ORIENTED, MAT_NEW_NONZERO_LOCATIONS, MAT_SYMMETRIC, MAT_STRUCTURALLY_SYMMETRIC,
  MAT_NEW_DIAGONALS, MAT_IGNORE_OFF_PROC_ENTRIES, MAT_USE_HASH_TABLE, MAT_KEEP_NONZERO_PATTERN,
  MAT_IGNORE_ZERO_ENTRIES, MAT_NEW_NONZERO_LOCATION_ERR, MAT_NEW_NONZERO_ALLOCATION_ERR,
  MAT_SPD, MAT_HERMITIAN, MAT_SYMMETRY_ETERNAL
} MatOption;
typedef int SNESConvergedReason;
typedef int KSPConvergedReason;

#define PETSC_NULL 0
#define PETSC_DEFAULT (-2)
#define PETSC_DECIDE (-1)
#define PETSC_DETERMINE (-1)
#define PETSC_COMM_WORLD 1
#define PETSC_COMM_SELF 2
#define MATAIJ "aij"
#define MATSEQAIJ "seqaij"
#define MATMPIAIJ "mpiaij"
#define MATDENSE "dense"
#define MATSEQDENSE "seqdense"
#define MATMPIDENSE "mpidense"
#define KSPPREONLY "preonly"
#define KSPCG "cg"
#define KSPGMRES "gmres"
#define PCLU "lu"
#define PCCHOLESKY "cholesky"
#define PCJACOBI "jacobi"
#define PCSOR "sor"
#define PCGAMG "gamg"
#define PCHYPRE "hypre"
#define PCNONE "none"
#define MATSOLVERMUMPS "mumps"
#define MATSOLVERSUPERLU_DIST "superlu_dist"
#define MATORDERINGND "nd"
#define MATORDERINGNATURAL "natural"
#define SNESNEWTONLS "newtonls"
#define SNESNEWTONTR "newtontr"
#define CHKERRQ(e) do { if (e) return (e); } while (0)
#define CHKERRV(e) do { if (e) return; } while (0)
#define CHKERRABORT(c, e) do { if (e) abort(); } while (0)
#define SETERRQ(c, n, s) return (n)
#define PETSC_ERR_ARG_WRONG 62

PetscErrorCode PetscInitialize(int* argc, char*** args, const char* file, const char* help);
PetscErrorCode PetscFinalize(void);
PetscErrorCode PetscPrintf(MPI_Comm comm, const char* fmt, ...);

PetscErrorCode MatCreate(MPI_Comm comm, Mat* A);
PetscErrorCode MatSetSizes(Mat A, PetscInt m, PetscInt n, PetscInt M, PetscInt N);
PetscErrorCode MatSetType(Mat A, MatType t);
PetscErrorCode MatSetFromOptions(Mat A);
PetscErrorCode MatSetUp(Mat A);
PetscErrorCode MatCreateSeqAIJ(MPI_Comm comm, PetscInt m, PetscInt n, PetscInt nz, const PetscInt nnz[], Mat* A);
PetscErrorCode MatCreateSeqDense(MPI_Comm comm, PetscInt m, PetscInt n, PetscScalar* data, Mat* A);
PetscErrorCode MatCreateDense(MPI_Comm comm, PetscInt m, PetscInt n, PetscInt M, PetscInt N, PetscScalar* data, Mat* A);
PetscErrorCode MatMPIAIJSetPreallocation(Mat B, PetscInt d_nz, const PetscInt d_nnz[], PetscInt o_nz, const PetscInt o_nnz[]);
PetscErrorCode MatSetBlockSize(Mat A, PetscInt bs);
PetscErrorCode MatSetOption(Mat A, MatOption op, PetscBool flg);
PetscErrorCode MatSetValue(Mat A, PetscInt i, PetscInt j, PetscScalar v, InsertMode mode);
PetscErrorCode MatSetValues(Mat A, PetscInt m, const PetscInt idxm[], PetscInt n, const PetscInt idxn[], const PetscScalar v[], InsertMode mode);
PetscErrorCode MatAssemblyBegin(Mat A, MatAssemblyType t);
PetscErrorCode MatAssemblyEnd(Mat A, MatAssemblyType t);
PetscErrorCode MatZeroEntries(Mat A);
PetscErrorCode MatSeqAIJGetArray(Mat A, PetscScalar** a);
PetscErrorCode MatSeqAIJRestoreArray(Mat A, PetscScalar** a);
PetscErrorCode MatMult(Mat A, Vec x, Vec y);
PetscErrorCode MatMultTranspose(Mat A, Vec x, Vec y);
PetscErrorCode MatGetOwnershipRange(Mat A, PetscInt* m, PetscInt* n);
PetscErrorCode MatGetOwnershipRangeColumn(Mat A, PetscInt* m, PetscInt* n);
PetscErrorCode MatGetOrdering(Mat A, MatOrderingType t, IS* rperm, IS* cperm);
PetscErrorCode MatGetFactor(Mat A, MatSolverPackage p, MatFactorType t, Mat* F);
PetscErrorCode MatCholeskyFactorSymbolic(Mat F, Mat A, IS perm, const MatFactorInfo* info);
PetscErrorCode MatCholeskyFactorNumeric(Mat F, Mat A, const MatFactorInfo* info);
PetscErrorCode MatMatSolve(Mat F, Mat B, Mat X);
PetscErrorCode MatGetColumnVector(Mat A, Vec y, PetscInt col);
PetscErrorCode MatDestroy(Mat* A);

PetscErrorCode VecCreateSeq(MPI_Comm comm, PetscInt n, Vec* v);
PetscErrorCode VecCreateMPI(MPI_Comm comm, PetscInt n, PetscInt N, Vec* v);
PetscErrorCode VecDuplicate(Vec v, Vec* newv);
PetscErrorCode VecSetValue(Vec v, PetscInt i, PetscScalar a, InsertMode mode);
PetscErrorCode VecSetValues(Vec v, PetscInt n, const PetscInt ix[], const PetscScalar y[], InsertMode mode);
PetscErrorCode VecGetValues(Vec v, PetscInt n, const PetscInt ix[], PetscScalar y[]);
PetscErrorCode VecAssemblyBegin(Vec v);
PetscErrorCode VecAssemblyEnd(Vec v);
PetscErrorCode VecZeroEntries(Vec v);
PetscErrorCode VecSet(Vec v, PetscScalar a);
PetscErrorCode VecAXPY(Vec y, PetscScalar a, Vec x);
PetscErrorCode VecCopy(Vec x, Vec y);
PetscErrorCode VecScale(Vec x, PetscScalar a);
PetscErrorCode VecDot(Vec x, Vec y, PetscScalar* val);
PetscErrorCode VecNorm(Vec x, NormType t, PetscReal* val);
PetscErrorCode VecGetArray(Vec x, PetscScalar** a);
PetscErrorCode VecRestoreArray(Vec x, PetscScalar** a);
PetscErrorCode VecGetArrayRead(Vec x, const PetscScalar** a);
PetscErrorCode VecRestoreArrayRead(Vec x, const PetscScalar** a);
PetscErrorCode VecGetOwnershipRange(Vec x, PetscInt* low, PetscInt* high);
PetscErrorCode VecGetSize(Vec x, PetscInt* n);
PetscErrorCode VecGetLocalSize(Vec x, PetscInt* n);
PetscErrorCode VecDestroy(Vec* v);
PetscErrorCode VecScatterCreate(Vec x, IS ix, Vec y, IS iy, VecScatter* ctx);
PetscErrorCode VecScatterCreateToAll(Vec x, VecScatter* ctx, Vec* y);
PetscErrorCode VecScatterBegin(VecScatter ctx, Vec x, Vec y, InsertMode addv, ScatterMode mode);
PetscErrorCode VecScatterEnd(VecScatter ctx, Vec x, Vec y, InsertMode addv, ScatterMode mode);
PetscErrorCode VecScatterDestroy(VecScatter* ctx);

PetscErrorCode ISCreateGeneral(MPI_Comm comm, PetscInt n, const PetscInt idx[], PetscCopyMode mode, IS* is);
PetscErrorCode ISDestroy(IS* is);

PetscErrorCode KSPCreate(MPI_Comm comm, KSP* ksp);
PetscErrorCode KSPSetOperators(KSP ksp, Mat A, Mat P);
PetscErrorCode KSPGetPC(KSP ksp, PC* pc);
PetscErrorCode KSPSetType(KSP ksp, KSPType t);
PetscErrorCode KSPCGSetType(KSP ksp, KSPCGType t);
PetscErrorCode KSPSetTolerances(KSP ksp, PetscReal rtol, PetscReal abstol, PetscReal dtol, PetscInt maxits);
PetscErrorCode KSPSetFromOptions(KSP ksp);
PetscErrorCode KSPSetUp(KSP ksp);
PetscErrorCode KSPSolve(KSP ksp, Vec b, Vec x);
PetscErrorCode KSPSolveTranspose(KSP ksp, Vec b, Vec x);
PetscErrorCode KSPGetIterationNumber(KSP ksp, PetscInt* its);
PetscErrorCode KSPDestroy(KSP* ksp);
PetscErrorCode PCSetType(PC pc, PCType t);
PetscErrorCode PCFactorSetMatSolverPackage(PC pc, MatSolverPackage p);
PetscErrorCode PCSetCoordinates(PC pc, PetscInt dim, PetscInt n, PetscReal* coords);
PetscErrorCode PCHYPRESetType(PC pc, const char* name);

PetscErrorCode SNESCreate(MPI_Comm comm, SNES* snes);
PetscErrorCode SNESSetType(SNES snes, SNESType t);
PetscErrorCode SNESSetFunction(SNES snes, Vec r, PetscErrorCode (*f)(SNES, Vec, Vec, void*), void* ctx);
PetscErrorCode SNESSetJacobian(SNES snes, Mat A, Mat P, PetscErrorCode (*J)(SNES, Vec, Mat, Mat, void*), void* ctx);
PetscErrorCode SNESMonitorSet(SNES snes, PetscErrorCode (*f)(SNES, PetscInt, PetscReal, void*), void* ctx, PetscErrorCode (*d)(void**));
PetscErrorCode SNESSetTolerances(SNES snes, PetscReal abstol, PetscReal rtol, PetscReal stol, PetscInt maxit, PetscInt maxf);
PetscErrorCode SNESGetKSP(SNES snes, KSP* ksp);
PetscErrorCode SNESSetFromOptions(SNES snes);
PetscErrorCode SNESSolve(SNES snes, Vec b, Vec x);
PetscErrorCode SNESGetFunctionNorm(SNES snes, PetscReal* norm);
PetscErrorCode SNESGetConvergedReason(SNES snes, SNESConvergedReason* r);
PetscErrorCode SNESDestroy(SNES* snes);

/* ------------------------------------------------------------------ GSL */
#define GSL_SUCCESS 0
#define GSL_FAILURE (-1)
#define GSL_CONTINUE (-2)
#define GSL_EDOM 1
#define GSL_EBADFUNC 9
#define GSL_EZERODIV 12
#define GSL_ENOPROG 27
#define GSL_ENOPROGJ 28
#define M_PI_SHIM 3.14159265358979323846

typedef struct { size_t size; size_t stride; double* data; void* block; int owner; } gsl_vector;
typedef struct { size_t size1; size_t size2; size_t tda; double* data; void* block; int owner; } gsl_matrix;
typedef struct { gsl_matrix matrix; } gsl_matrix_view;
typedef struct { double (*function)(double x, void* params); void* params; } gsl_function;
typedef struct {
  double (*f)(double x, void* params);
  double (*df)(double x, void* params);
  void (*fdf)(double x, void* params, double* f, double* df);
  void* params;
} gsl_function_fdf;

gsl_vector* gsl_vector_alloc(size_t n);
gsl_vector* gsl_vector_calloc(size_t n);
void gsl_vector_free(gsl_vector* v);
double gsl_vector_get(const gsl_vector* v, size_t i);
void gsl_vector_set(gsl_vector* v, size_t i, double x);
gsl_matrix* gsl_matrix_alloc(size_t n1, size_t n2);
void gsl_matrix_free(gsl_matrix* m);
double gsl_matrix_get(const gsl_matrix* m, size_t i, size_t j);
void gsl_matrix_set(gsl_matrix* m, size_t i, size_t j, double x);
gsl_matrix_view gsl_matrix_view_array(double* base, size_t n1, size_t n2);

typedef struct pg_root_fsolver_type { const char* name; } gsl_root_fsolver_type;
typedef struct pg_root_fdfsolver_type { const char* name; } gsl_root_fdfsolver_type;
typedef struct pg_root_fsolver gsl_root_fsolver;
typedef struct pg_root_fdfsolver gsl_root_fdfsolver;
extern const gsl_root_fsolver_type* gsl_root_fsolver_brent;
extern const gsl_root_fsolver_type* gsl_root_fsolver_bisection;
extern const gsl_root_fdfsolver_type* gsl_root_fdfsolver_steffenson;
extern const gsl_root_fdfsolver_type* gsl_root_fdfsolver_newton;
gsl_root_fsolver* gsl_root_fsolver_alloc(const gsl_root_fsolver_type* T);
int gsl_root_fsolver_set(gsl_root_fsolver* s, gsl_function* f, double x_lower, double x_upper);
int gsl_root_fsolver_iterate(gsl_root_fsolver* s);
double gsl_root_fsolver_root(const gsl_root_fsolver* s);
double gsl_root_fsolver_x_lower(const gsl_root_fsolver* s);
double gsl_root_fsolver_x_upper(const gsl_root_fsolver* s);
void gsl_root_fsolver_free(gsl_root_fsolver* s);
gsl_root_fdfsolver* gsl_root_fdfsolver_alloc(const gsl_root_fdfsolver_type* T);
int gsl_root_fdfsolver_set(gsl_root_fdfsolver* s, gsl_function_fdf* fdf, double root);
int gsl_root_fdfsolver_iterate(gsl_root_fdfsolver* s);
double gsl_root_fdfsolver_root(const gsl_root_fdfsolver* s);
void gsl_root_fdfsolver_free(gsl_root_fdfsolver* s);
int gsl_root_test_delta(double x1, double x0, double epsabs, double epsrel);
int gsl_root_test_interval(double x_lower, double x_upper, double epsabs, double epsrel);

typedef struct {
  int (*f)(const gsl_vector* x, void* params, gsl_vector* f);
  int (*df)(const gsl_vector* x, void* params, gsl_matrix* df);
  int (*fdf)(const gsl_vector* x, void* params, gsl_vector* f, gsl_matrix* df);
  size_t n;
  void* params;
} gsl_multiroot_function_fdf;
typedef struct pg_multiroot_fdfsolver_type { const char* name; } gsl_multiroot_fdfsolver_type;
typedef struct {
  const gsl_multiroot_fdfsolver_type* type;
  gsl_multiroot_function_fdf* fdf;
  gsl_vector* x;
  gsl_vector* f;
  gsl_matrix* J;
  gsl_vector* dx;
  void* state;
} gsl_multiroot_fdfsolver;
extern const gsl_multiroot_fdfsolver_type* gsl_multiroot_fdfsolver_hybridj;
extern const gsl_multiroot_fdfsolver_type* gsl_multiroot_fdfsolver_hybridsj;
extern const gsl_multiroot_fdfsolver_type* gsl_multiroot_fdfsolver_newton;
gsl_multiroot_fdfsolver* gsl_multiroot_fdfsolver_alloc(const gsl_multiroot_fdfsolver_type* T, size_t n);
int gsl_multiroot_fdfsolver_set(gsl_multiroot_fdfsolver* s, gsl_multiroot_function_fdf* fdf, const gsl_vector* x);
int gsl_multiroot_fdfsolver_iterate(gsl_multiroot_fdfsolver* s);
void gsl_multiroot_fdfsolver_free(gsl_multiroot_fdfsolver* s);
int gsl_multiroot_test_residual(const gsl_vector* f, double epsabs);

typedef struct pg_eigen_symm_workspace gsl_eigen_symm_workspace;
gsl_eigen_symm_workspace* gsl_eigen_symm_alloc(size_t n);
int gsl_eigen_symm(gsl_matrix* A, gsl_vector* eval, gsl_eigen_symm_workspace* w);
void gsl_eigen_symm_free(gsl_eigen_symm_workspace* w);

enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
typedef enum CBLAS_ORDER CBLAS_ORDER_t;
typedef enum CBLAS_TRANSPOSE CBLAS_TRANSPOSE_t;
void cblas_daxpy(const int N, const double alpha, const double* X, const int incX, double* Y, const int incY);
void cblas_saxpy(const int N, const float alpha, const float* X, const int incX, float* Y, const int incY);
void cblas_dscal(const int N, const double alpha, double* X, const int incX);
void cblas_sscal(const int N, const float alpha, float* X, const int incX);
double cblas_ddot(const int N, const double* X, const int incX, const double* Y, const int incY);
void cblas_dgemv(const enum CBLAS_ORDER order, const enum CBLAS_TRANSPOSE TransA, const int M, const int N,
                 const double alpha, const double* A, const int lda, const double* X, const int incX,
                 const double beta, double* Y, const int incY);
void cblas_sgemv(const enum CBLAS_ORDER order, const enum CBLAS_TRANSPOSE TransA, const int M, const int N,
                 const float alpha, const float* A, const int lda, const float* X, const int incX,
                 const float beta, float* Y, const int incY);
void cblas_dgemm(const enum CBLAS_ORDER Order, const enum CBLAS_TRANSPOSE TransA, const enum CBLAS_TRANSPOSE TransB,
                 const int M, const int N, const int K, const double alpha, const double* A, const int lda,
                 const double* B, const int ldb, const double beta, double* C, const int ldc);
void cblas_sgemm(const enum CBLAS_ORDER Order, const enum CBLAS_TRANSPOSE TransA, const enum CBLAS_TRANSPOSE TransB,
                 const int M, const int N, const int K, const float alpha, const float* A, const int lda,
                 const float* B, const int ldb, const float beta, float* C, const int ldc);

#ifdef __cplusplus
}
#endif
