// pg_ctx.h -- the context behind the C ABI's opaque pg_ctx (internal to libpigfem_b200).
//
// A pg_ctx owns every device buffer of one problem: geometry, topology, the cut-element
// quadrature tables, the CSR structure and values of the four blocks, the residual, the
// committed and trial internal variables, the cut-element scratch and the solver workspace.
#pragma once

#include "pg_stencil.cuh"
#include "pg_setup.h"
#include "../../include/pigfem_b200.h"

#include <string>
#include <vector>

namespace pgd { struct Tile3Const; }

// Workspace of the Jacobi-preconditioned CG on K_ff (pg_solver.cu), allocated on first use.
struct PcgWork {
  int n = 0, cap_rhs = 0, nb = 0;
  double* dinv = nullptr;                       // n: inverse diagonal of K_ff
  const int* ci = nullptr;                      // column indices of K_ff
  double *r = nullptr, *z = nullptr, *p = nullptr, *q = nullptr;  // cap_rhs x n each
  double* part = nullptr;                       // partial sums: 3 x cap_rhs x nb
  double* sc = nullptr;                         // scalars per rhs (see pg_solver.cu)
  int* flag = nullptr;                          // per rhs: done, iterations; [2*cap_rhs] = active count
  int* hflag = nullptr;                         // pinned host copy of flag
  cudaStream_t stream = nullptr;
  cudaEvent_t ev = nullptr;
  bool diag_ready = false;
};

struct pg_ctx {
  pg::Setup s;
  std::string err;
  cudaStream_t stream = 0;
  std::vector<void*> allocs;
  std::vector<size_t> alloc_bytes;   // bytes of allocs[i]
  size_t dev_bytes = 0, dev_bytes_peak = 0;   // held now / most held at once (pg_device_bytes)
  pgd::DevProblem P{};
  double* d_U = nullptr;
  double* d_isv_committed = nullptr;
  double* d_isv_trial = nullptr;
  uint8_t* d_zone = nullptr;
  int* d_err = nullptr;
  double* d_red = nullptr;  // residual-norm partials
  long long cut_scratch = 0;   // doubles of the cut elements' set-up blocks (released after set-up)
  long long stat_doubles = 0;  // doubles of the general rows' static part
  int max_nd = 0;
  int maxnb_fast = 0;
  int n_coh_qp = 0;
  bool assembled = false;
  pgd::Tile3Const* t3c = nullptr;         // 3D tiles' shape constants: host copy (kernel parameter)
  const pgd::Tile3Const* d_t3c = nullptr; // and device copy (batches)
  bool timed_last = false;   // the last assembly recorded every timing event (pg_kernel_times)
  double prep_ms = -1.0;   // device time of the preprocessing passes (pg_create_prep_device), -1 if none ran
  // PG_KEEP_STATIC: the first CSR value of each block from which a later assembly can change
  // values (the rows of DOFs of nodes on cohesive elements; nnz when no value can change), and
  // the host arrays (and precision) the last full copy of K went to
  long long changing_from[4] = {0, 0, 0, 0};
  double* kept[4] = {nullptr, nullptr, nullptr, nullptr};
  bool kept_fp32 = false, kept_valid = false;
  std::vector<int> fast_dn, slow_dn;
  int tile_nodes = 128;
  int max_cut_qp = 1, max_cut_nodes = 1;
  const int* cut_list[2] = {nullptr, nullptr};
  int n_cut_list[2] = {0, 0};
  int cut_cls_qp[2] = {1, 1}, cut_cls_nodes[2] = {1, 1};
  const int4* stencil = nullptr;
  int n_stencil = 0;
  // 2D tiles of the stencil rows (pg_tile.cuh): per tile {i0, j0, first segment, segments}, per
  // tile 128 node entries {node, first DOF, first CSR slot, stage offset}, the store segments
  const int4* tiles = nullptr;
  const int4* tnodes = nullptr;
  const int4* tsegs = nullptr;
  int n_tiles = 0;
  pgd::GridInfo grid{0, 0, 0};
  bool timing = false;
  cudaStream_t side = nullptr;    // 2D: the structured tiles (lowest stream priority)
  cudaStream_t side2 = nullptr;   // 2D: cohesive elements, records and general rows (highest priority)
  // fork, tiles done, (unused), first kernel done, general rows done, join
  cudaEvent_t ev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  PcgWork pcg;
  // material sensitivity pass (pg_sens.cu): made on its first call
  struct SensWork {
    bool ready = false;
    double* uncut = nullptr;   // per element: NPE x DIM values
    double* cut = nullptr;     // per cut-element node: DIM values
    double* dD = nullptr;      // 2 materials x 5 parameters x 36
    double* g = nullptr;       // the cut elements' point gradients (unmerged)
    int* g_off = nullptr;
    int* pt_off = nullptr;     // a call's point lists
    double* pt_w = nullptr;
    int* pt_g = nullptr;
  } sens;
  double* d_hom = nullptr;  // homogenization partials
  // Device memory comes from the stream-ordered pool on this stream (cudaMallocAsync /
  // cudaFreeAsync): creating and destroying contexts does not synchronise the device, so other
  // contexts' work in flight (the serving loop) keeps running.
  cudaStream_t up = nullptr;
};

// Whether the context's tables are on the device (pg_create, or pg_create_host then pg_upload);
// every entry point that launches work checks it first, so a host-only context gets
// PG_ERR_STATE instead of kernels on null pointers.
inline bool pg_resident(const pg_ctx* c) { return c && c->P.X != nullptr && c->d_err != nullptr; }

// The allocation stream of a context (created on first use).
int pg_alloc_stream(pg_ctx* c);

// Shared helpers of the translation units of the library.
int pg_set_err(pg_ctx* c, int code, const std::string& m);
// Record a device allocation of the context (freed by pg_destroy, or earlier by pg_untrack_free).
inline void pg_track_alloc(pg_ctx* c, void* p, size_t bytes) {
  c->allocs.push_back(p);
  c->alloc_bytes.push_back(bytes);
  c->dev_bytes += bytes;
  if (c->dev_bytes > c->dev_bytes_peak) c->dev_bytes_peak = c->dev_bytes;
}
// Free one tracked allocation early (stream-ordered on the allocation stream).
inline void pg_untrack_free(pg_ctx* c, void* p) {
  for (size_t i = 0; i < c->allocs.size(); ++i)
    if (c->allocs[i] == p) {
      c->dev_bytes -= c->alloc_bytes[i];
      c->allocs.erase(c->allocs.begin() + i);
      c->alloc_bytes.erase(c->alloc_bytes.begin() + i);
      cudaFreeAsync(p, c->up);
      return;
    }
}

// Zero-filled device array of n T on the context's allocation stream; ready for other streams
// after pg_alloc_sync(c).
template <typename T>
int pg_dalloc(pg_ctx* c, size_t n, T** out) {
  *out = nullptr;
  if (n == 0) n = 1;
  if (int rc = pg_alloc_stream(c)) return rc;
  void* p = nullptr;
  if (cudaMallocAsync(&p, n * sizeof(T), c->up) != cudaSuccess) return pg_set_err(c, PG_ERR_DEVICE, "device allocation failed");
  pg_track_alloc(c, p, n * sizeof(T));
  cudaMemsetAsync(p, 0, n * sizeof(T), c->up);
  *out = (T*)p;
  return 0;
}
int pg_alloc_sync(pg_ctx* c);


