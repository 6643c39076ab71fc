// pg_batch.cu -- many RVEs in one set of persistent launches, replayed from a CUDA graph.
//
// A batch holds the device descriptors (DevProblem) of n assembled-ready contexts and three work
// lists that cover all of them: chunks of cohesive elements, of structured stencil nodes and of
// general DOF nodes, each chunk {context, first item, count}.  One assembly of the whole batch is
// three persistent kernels (cohesive elements and general rows on the batch stream, stencil rows
// concurrently on a side stream) that stride over the chunk lists; the whole sequence, including
// the upload of the per-call parameters (each context's displacement pointer, flags and
// macroscale strain), is captured once into a CUDA graph and replayed.  Every CSR value and
// residual entry is still written by exactly one thread group with the same arithmetic as the
// single-context launches, so each context's results are bitwise those of pg_assemble_device.
//
// The autotuner (pg_batch_tune) times the candidate launch shapes on the batch itself and keeps
// the fastest: stencil nodes per block (64 / 128 / 256), general-row lanes per node (2D: 4 / 8 / 16,
// 3D: 8 / 16 / 32) and the persistent grid (2 / 4 / 8 blocks per SM).
#include "pg_ctx.h"
#include "pg_tile.cuh"
#include "pg_general.cuh"

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

namespace {

struct BatchItem {
  pgd::DevProblem P;
  pgd::GridInfo gi;
  const int4* stencil;
  int n_stencil;
  const int4* tiles;    // 2D: the context's stencil tiles (pg_tile.cuh)
  const int4* tnodes;
  const int4* tsegs;
  const pgd::Tile3Const* t3c;   // 3D: the context's tile shape constants (device copy)
};

struct BatchCall {
  const double* U;
  int flags;
  int pad;
  double eps[6];
};

constexpr int kSMs = 148;

__global__ void k_batch_prepare(BatchItem* items, const BatchCall* call, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    items[i].P.U = call[i].U;
    items[i].P.flags = call[i].flags;
    for (int v = 0; v < 6; ++v) items[i].P.eps_macro[v] = call[i].eps[v];
    *items[i].P.err = 0;
  }
}

__global__ void k_batch_errors(const BatchItem* items, int n, int* out) {
  int e = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) e |= *items[i].P.err;
  e = __reduce_or_sync(0xffffffffu, e);
  if ((threadIdx.x & 31) == 0 && e) atomicOr(out, e);
}

// chunk = 128 / CQ cohesive elements, CQ lanes each
template <int DIM>
__global__ void __launch_bounds__(128) k_batch_coh(const BatchItem* __restrict__ items, const int4* __restrict__ chunks,
                                                   int n_chunks) {
  constexpr int CQ = pgd::CohLanes<DIM>::CQ;
  const int e = threadIdx.x / CQ, qi = threadIdx.x % CQ;
  for (int c = blockIdx.x; c < n_chunks; c += gridDim.x) {
    const int4 ch = chunks[c];
    pgd::coh_element<DIM>(items[ch.x].P, ch.y + e, qi, e < ch.z);
  }
}

// One CTA per stencil tile (chunk = one tile): 2D the body of k_rows_tile2 (256 threads), 3D that
// of k_rows_tile3 (192 threads).
template <int DIM, typename T>
__global__ void __launch_bounds__(256) k_batch_stencil(const BatchItem* __restrict__ items, const int4* __restrict__ chunks,
                                                       int n_chunks) {
  extern __shared__ double stage[];
  for (int c = blockIdx.x; c < n_chunks; c += gridDim.x) {
    const int4 ch = chunks[c];
    const BatchItem& it = items[ch.x];
    if (DIM == 2) {
      pgd::stencil_tile2<T, true>(it.P, it.gi, __ldg(&it.tiles[ch.y]), it.tnodes + (size_t)ch.y * pgd::kTileOwn,
                                  it.tsegs, stage);
      __syncthreads();
    } else {
      pgd::stencil_tile3<T, true>(it.P, it.gi, __ldg(&it.tiles[2 * ch.y]), __ldg(&it.tiles[2 * ch.y + 1]),
                                  it.tnodes + (size_t)ch.y * pgd::kT3Nodes, it.tsegs, stage, *it.t3c);
      __syncthreads();
    }
  }
}

// The block-parallel general rows (pg_general.cuh) of every context: chunk = {context, first
// item, count <= 128, pass} with pass 1 blocks, 2 residuals (pass 0, element records, has no
// chunks: the general rows read their static image); the passes are launches in that order.
template <int DIM>
__global__ void __launch_bounds__(128) k_batch_gen(const BatchItem* __restrict__ items, const int4* __restrict__ chunks,
                                                  int n_chunks) {
  for (int c = blockIdx.x; c < n_chunks; c += gridDim.x) {
    const int4 ch = chunks[c];
    const pgd::DevProblem& P = items[ch.x].P;
    if (ch.w == 2) {   // residuals: a group of kGenResidLanes lanes per node, 128 / lanes nodes per chunk
      const int grp = threadIdx.x / pgd::kGenResidLanes;
      if (P.flags & pgd::FLAG_FUNC) pgd::gen_resid<DIM, pgd::kGenResidLanes>(P, ch.y + grp, grp < ch.z);
      continue;
    }
    if ((int)threadIdx.x >= ch.z) continue;
    const int k = ch.y + threadIdx.x;
    if (ch.w == 1 && (P.flags & pgd::FLAG_JAC)) pgd::gen_block<DIM>(P, k);
  }
}

}  // namespace

struct pg_batch {
  std::vector<pg_ctx*> ctx;
  int dim = 2;
  BatchItem* d_items = nullptr;
  BatchCall* d_call = nullptr;
  BatchCall* h_call = nullptr;
  int4 *d_coh = nullptr, *d_sten = nullptr, *d_gen[3] = {nullptr, nullptr, nullptr};
  int* d_err = nullptr;   // OR of the contexts' device error words of the last call
  int n_coh = 0, n_sten = 0, n_gen[3] = {0, 0, 0};   // general rows: records, blocks, residuals
  int max_mn = 1;
  int mult = 4;   // launch shape (autotuned): persistent blocks per SM
  cudaStream_t stream = nullptr, side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr, t0 = nullptr, t1 = nullptr;
  cudaGraphExec_t exec[2] = {nullptr, nullptr};   // FP64, FP32-mixed
  bool launched = false;
  long long n_elem = 0;
  std::string err;
};

namespace {

int berr(pg_batch* b, int code, const std::string& m) {
  if (b) b->err = m;
  return code;
}

void free_chunks(pg_batch* b) {
  if (b->d_coh) cudaFree(b->d_coh);
  if (b->d_sten) cudaFree(b->d_sten);
  for (int k = 0; k < 3; ++k) { if (b->d_gen[k]) cudaFree(b->d_gen[k]); b->d_gen[k] = nullptr; }
  b->d_coh = b->d_sten = nullptr;
}

void drop_graphs(pg_batch* b) {
  for (auto& e : b->exec)
    if (e) { cudaGraphExecDestroy(e); e = nullptr; }
}

template <typename T>
int upload_vec(pg_batch* b, const std::vector<T>& h, T** d) {
  *d = nullptr;
  if (h.empty()) return 0;
  if (cudaMalloc(d, h.size() * sizeof(T)) != cudaSuccess) return berr(b, PG_ERR_DEVICE, "cudaMalloc failed");
  if (cudaMemcpy(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
    return berr(b, PG_ERR_DEVICE, "cudaMemcpy failed");
  return 0;
}

// set before any capture: the dynamic shared memory of the kernels of the current shape
void set_attributes(const pg_batch* b) {
  cudaFuncSetAttribute(k_batch_stencil<2, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pgd::tile2_smem_bytes());
  cudaFuncSetAttribute(k_batch_stencil<2, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pgd::tile2_smem_bytes());
  cudaFuncSetAttribute(k_batch_stencil<3, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pgd::tile3_smem_bytes());
  cudaFuncSetAttribute(k_batch_stencil<3, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pgd::tile3_smem_bytes());
}

// Chunk lists for the current launch shape.
int build_chunks(pg_batch* b) {
  free_chunks(b);
  drop_graphs(b);
  std::vector<int4> coh, sten, gen[3];

  for (int i = 0; i < (int)b->ctx.size(); ++i) {
    const pg_ctx* c = b->ctx[i];
    const int coh_chunk = 128 / ((b->dim == 2) ? pgd::CohLanes<2>::CQ : pgd::CohLanes<3>::CQ);
    for (int f = 0; f < c->P.n_coh_el; f += coh_chunk)
      coh.push_back(make_int4(i, f, std::min(coh_chunk, c->P.n_coh_el - f), 0));
    for (int tl = 0; tl < c->n_tiles; ++tl) sten.push_back(make_int4(i, tl, 1, 0));
    const int ng[3] = {0, c->P.n_gblk, c->P.n_slow_dn};
    for (int pass = 0; pass < 3; ++pass)
      for (int f = 0, per = (pass == 2) ? 128 / pgd::kGenResidLanes : 128; f < ng[pass]; f += per)
        gen[pass].push_back(make_int4(i, f, std::min(per, ng[pass] - f), pass));
  }
  b->n_coh = (int)coh.size();
  b->n_sten = (int)sten.size();
  for (int k = 0; k < 3; ++k) b->n_gen[k] = (int)gen[k].size();
  int rc = upload_vec(b, coh, &b->d_coh);
  rc = rc ? rc : upload_vec(b, sten, &b->d_sten);
  for (int k = 0; k < 3; ++k) rc = rc ? rc : upload_vec(b, gen[k], &b->d_gen[k]);
  if (!rc) set_attributes(b);
  return rc;
}


void enqueue(pg_batch* b, bool fp32) {
  const int nb = (int)b->ctx.size();
  cudaStream_t st = b->stream;
  cudaMemcpyAsync(b->d_call, b->h_call, sizeof(BatchCall) * nb, cudaMemcpyHostToDevice, st);
  cudaMemsetAsync(b->d_err, 0, sizeof(int), st);
  k_batch_prepare<<<(nb + 127) / 128, 128, 0, st>>>(b->d_items, b->d_call, nb);
  cudaEventRecord(b->fork, st);
  cudaStreamWaitEvent(b->side, b->fork, 0);
  const int cap = b->mult * kSMs;
  if (b->n_coh) {
    const int grid = std::min(b->n_coh, cap);
    if (b->dim == 2) k_batch_coh<2><<<grid, 128, 0, st>>>(b->d_items, b->d_coh, b->n_coh);
    else k_batch_coh<3><<<grid, 128, 0, st>>>(b->d_items, b->d_coh, b->n_coh);
  }
  if (b->n_sten) {
    const int grid = std::min(b->n_sten, cap);
    if (b->dim == 2) {
      const size_t smem = pgd::tile2_smem_bytes();
      if (fp32) k_batch_stencil<2, float><<<grid, pgd::kTileThreads, smem, b->side>>>(b->d_items, b->d_sten, b->n_sten);
      else k_batch_stencil<2, double><<<grid, pgd::kTileThreads, smem, b->side>>>(b->d_items, b->d_sten, b->n_sten);
    } else {
      const size_t smem = pgd::tile3_smem_bytes();
      if (fp32) k_batch_stencil<3, float><<<grid, pgd::kT3Threads, smem, b->side>>>(b->d_items, b->d_sten, b->n_sten);
      else k_batch_stencil<3, double><<<grid, pgd::kT3Threads, smem, b->side>>>(b->d_items, b->d_sten, b->n_sten);
    }
  }
  for (int pass = 0; pass < 3; ++pass) {
    if (!b->n_gen[pass]) continue;
    const int grid = std::min(b->n_gen[pass], cap);
    if (b->dim == 2) k_batch_gen<2><<<grid, 128, 0, st>>>(b->d_items, b->d_gen[pass], b->n_gen[pass]);
    else k_batch_gen<3><<<grid, 128, 0, st>>>(b->d_items, b->d_gen[pass], b->n_gen[pass]);
  }
  cudaEventRecord(b->join, b->side);
  cudaStreamWaitEvent(st, b->join, 0);
  k_batch_errors<<<1, 256, 0, st>>>(b->d_items, nb, b->d_err);
}

int graph_for(pg_batch* b, bool fp32, cudaGraphExec_t* out) {
  cudaGraphExec_t& e = b->exec[fp32 ? 1 : 0];
  if (!e) {
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
      return berr(b, PG_ERR_DEVICE, "graph capture failed to start");
    enqueue(b, fp32);
    if (cudaStreamEndCapture(b->stream, &g) != cudaSuccess) return berr(b, PG_ERR_DEVICE, "graph capture failed");
    const cudaError_t ie = cudaGraphInstantiate(&e, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) { e = nullptr; return berr(b, PG_ERR_DEVICE, "graph instantiation failed"); }
  }
  *out = e;
  return 0;
}

void fill_call(pg_batch* b, const double* const* d_U, const double* t_frac, int flags) {
  for (size_t i = 0; i < b->ctx.size(); ++i) {
    BatchCall& k = b->h_call[i];
    k.U = d_U[i];
    k.flags = flags & (PG_FUNC | PG_JAC);
    const double tf = t_frac ? t_frac[i] : 1.0;
    for (int v = 0; v < 6; ++v) k.eps[v] = b->ctx[i]->s.desc.eps_macro[v] * tf;
  }
}

}  // namespace

extern "C" {

int pg_batch_create(pg_ctx* const* ctxs, int n, pg_batch** out) {
  if (!ctxs || n < 1 || !out) return PG_ERR_INPUT;
  *out = nullptr;
  pg_batch* b = new pg_batch;
  *out = b;
  b->dim = ctxs[0] ? ctxs[0]->s.dim : 2;
  std::vector<BatchItem> items(n);
  for (int i = 0; i < n; ++i) {
    pg_ctx* c = ctxs[i];
    if (!c || !c->P.X) return berr(b, PG_ERR_INPUT, "every context must be uploaded (pg_create or pg_upload)");
    if (c->s.dim != b->dim) return berr(b, PG_ERR_INPUT, "a batch holds contexts of one dimension");
    if (c->s.etype == pg::QUAD4) return berr(b, PG_ERR_UNSUPPORTED, "batches take tri3 / tet4 contexts");
    b->ctx.push_back(c);
    items[i].P = c->P;
    items[i].gi = c->grid;
    items[i].stencil = c->stencil;
    items[i].n_stencil = c->n_stencil;
    items[i].tiles = c->tiles;
    items[i].tnodes = c->tnodes;
    items[i].tsegs = c->tsegs;
    items[i].t3c = c->d_t3c;
    b->max_mn = std::max(b->max_mn, c->P.max_mn);
    b->n_elem += c->s.ne;
  }
  if (cudaMalloc(&b->d_items, sizeof(BatchItem) * n) != cudaSuccess) return berr(b, PG_ERR_DEVICE, "cudaMalloc failed");
  cudaMemcpy(b->d_items, items.data(), sizeof(BatchItem) * n, cudaMemcpyHostToDevice);
  if (cudaMalloc(&b->d_err, sizeof(int)) != cudaSuccess || cudaMalloc(&b->d_call, sizeof(BatchCall) * n) != cudaSuccess ||
      cudaMallocHost(&b->h_call, sizeof(BatchCall) * n) != cudaSuccess)
    return berr(b, PG_ERR_DEVICE, "call-parameter buffers failed");
  std::memset(b->h_call, 0, sizeof(BatchCall) * n);
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking) != cudaSuccess)
    return berr(b, PG_ERR_DEVICE, "stream creation failed");
  cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
  cudaEventCreateWithFlags(&b->join, cudaEventDisableTiming);
  cudaEventCreate(&b->t0);
  cudaEventCreate(&b->t1);
  return build_chunks(b);
}

int pg_batch_assemble(pg_batch* b, const double* const* d_U, const double* t_frac, int flags) {
  if (!b || !d_U) return PG_ERR_INPUT;
  if (b->launched && cudaEventSynchronize(b->t1) != cudaSuccess) return berr(b, PG_ERR_DEVICE, "previous batch failed");
  for (size_t i = 0; i < b->ctx.size(); ++i) {
    if (!d_U[i]) return berr(b, PG_ERR_INPUT, "missing displacement pointer");
    if (reinterpret_cast<uintptr_t>(d_U[i]) % 16) return berr(b, PG_ERR_INPUT, "displacement arrays must be 16-byte aligned");
  }
  fill_call(b, d_U, t_frac, flags);
  cudaGraphExec_t e;
  if (int rc = graph_for(b, (flags & PG_FP32) != 0, &e)) return rc;
  cudaEventRecord(b->t0, b->stream);
  if (cudaGraphLaunch(e, b->stream) != cudaSuccess) return berr(b, PG_ERR_DEVICE, "graph launch failed");
  cudaEventRecord(b->t1, b->stream);
  b->launched = true;
  for (pg_ctx* c : b->ctx) c->assembled = true;
  return 0;
}

int pg_batch_wait(pg_batch* b, float* ms) {
  if (!b) return PG_ERR_INPUT;
  if (!b->launched) return berr(b, PG_ERR_STATE, "nothing was launched");
  if (cudaEventSynchronize(b->t1) != cudaSuccess) return berr(b, PG_ERR_DEVICE, "batch assembly failed");
  if (ms) cudaEventElapsedTime(ms, b->t0, b->t1);
  int herr = 0;
  cudaMemcpy(&herr, b->d_err, sizeof(int), cudaMemcpyDeviceToHost);
  if (herr) return berr(b, (herr & pgd::ERR_NONFINITE) ? PG_ERR_NONFINITE : PG_ERR_DEVICE,
                        "a context of the batch reported a device error (pg_last_error of each context has no detail)");
  return 0;
}

int pg_batch_tune(pg_batch* b, const double* const* d_U, int flags, int reps, int* best) {
  if (!b || !d_U || reps < 1) return PG_ERR_INPUT;
  const int mults[4] = {2, 4, 8, 16};
  float best_ms = 1e30f;
  int bm = b->mult;
  for (int mi = 0; mi < 4; ++mi) {
    b->mult = mults[mi];
    if (int rc = build_chunks(b)) return rc;
    float total = 0.0f;
    for (int r = 0; r < reps + 2; ++r) {
      if (int rc = pg_batch_assemble(b, d_U, nullptr, flags)) return rc;
      float ms = 0.0f;
      if (int rc = pg_batch_wait(b, &ms)) return rc;
      if (r >= 2) total += ms;
    }
    if (total < best_ms) { best_ms = total; bm = b->mult; }
  }
  b->mult = bm;
  if (best) { best[0] = (b->dim == 2) ? pgd::kTileThreads : pgd::kT3Threads; best[1] = 1; best[2] = bm; }
  return build_chunks(b);
}

int pg_batch_info(const pg_batch* b, int64_t* info) {
  if (!b || !info) return PG_ERR_INPUT;
  info[0] = (int64_t)b->ctx.size();
  info[1] = b->n_elem;
  info[2] = (b->dim == 2) ? pgd::kTileThreads : pgd::kT3Threads; info[3] = 1; info[4] = b->mult;
  info[5] = b->n_coh; info[6] = b->n_sten; info[7] = b->n_gen[0] + b->n_gen[1] + b->n_gen[2];
  return 0;
}

const char* pg_batch_last_error(const pg_batch* b) { return b ? b->err.c_str() : "null batch"; }

void pg_batch_destroy(pg_batch* b) {
  if (!b) return;
  if (b->launched) cudaEventSynchronize(b->t1);
  drop_graphs(b);
  free_chunks(b);
  if (b->d_items) cudaFree(b->d_items);
  if (b->d_call) cudaFree(b->d_call);
  if (b->d_err) cudaFree(b->d_err);
  if (b->h_call) cudaFreeHost(b->h_call);
  for (cudaEvent_t e : {b->fork, b->join, b->t0, b->t1}) if (e) cudaEventDestroy(e);
  if (b->stream) cudaStreamDestroy(b->stream);
  if (b->side) cudaStreamDestroy(b->side);
  delete b;
}

}  // extern "C"
