// pg_capi.cu -- the C ABI (include/pigfem_b200.h): set-up, device residency, launches.
//
// A pg_ctx owns every device buffer of one problem: geometry, topology, the cut-element
// quadrature tables, the CSR structure and values of the four blocks, the residual, the
// committed and trial internal variables and the cut-element scratch.  The caller owns its
// host arrays; pointers are never retained across calls.
#include "pg_ctx.h"
#include "pg_launch.cuh"
#include "pg_tile.cuh"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace {

int set_err(pg_ctx* c, int code, const std::string& m) { return pg_set_err(c, code, m); }

template <typename T>
int upload(pg_ctx* c, const std::vector<T>& h, const T** out) {
  *out = nullptr;
  if (h.empty()) return 0;
  if (int rc = pg_alloc_stream(c)) return rc;
  void* p = nullptr;
  if (cudaMallocAsync(&p, h.size() * sizeof(T), c->up) != cudaSuccess) return set_err(c, PG_ERR_DEVICE, "device allocation failed");
  pg_track_alloc(c, p, h.size() * sizeof(T));
  // pageable source: the call returns once the data is staged, so `h` may go away afterwards
  if (cudaMemcpyAsync(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, c->up) != cudaSuccess)
    return set_err(c, PG_ERR_DEVICE, "host-to-device copy failed");
  *out = (const T*)p;
  return 0;
}

template <typename T>
int dalloc(pg_ctx* c, size_t n, T** out) { return pg_dalloc(c, n, out); }

#define PG_TRY(x) do { int _e = (x); if (_e) return _e; } while (0)

// Fixed-order sum of squares: each block reduces a contiguous chunk in a fixed tree order.
__global__ void k_sumsq_partial(const double* x, int n, double* part) {
  __shared__ double sh[256];
  const int chunk = (n + gridDim.x - 1) / gridDim.x;
  const int b0 = blockIdx.x * chunk, b1 = min(n, b0 + chunk);
  double s = 0.0;
  for (int i = b0 + threadIdx.x; i < b1; i += blockDim.x) s += x[i] * x[i];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}
__global__ void k_sum_final(const double* part, int n, double* out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += part[i];
    out[0] = s;
  }
}

int launch(pg_ctx* c, double t_frac, int flags) {
  if (!c->ev[0])
    for (int i = 0; i < 6; ++i) cudaEventCreateWithFlags(&c->ev[i], cudaEventDefault);
  pgd::DevProblem P = c->P;
  P.U = c->d_U;
  P.flags = flags;
  for (int v = 0; v < 6; ++v) P.eps_macro[v] = c->s.desc.eps_macro[v] * t_frac;
  const int dim = c->s.dim;
  const bool fp32 = (flags & PG_FP32) != 0;
  const bool jac = (flags & PG_JAC) != 0;   // without it: the residual-only kernels
  if (dim == 2) pgl::assembly<2>(c, P, jac, fp32);
  else pgl::assembly<3>(c, P, jac, fp32);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_err(c, PG_ERR_DEVICE, std::string("launch failed: ") + cudaGetErrorString(e));
  return 0;
}

}  // namespace

int pg_set_err(pg_ctx* c, int code, const std::string& m) {
  if (c) c->err = m;
  return code;
}

int pg_alloc_stream(pg_ctx* c) {
  if (c->up) return 0;
  static bool pool_ready = false;
  if (!pool_ready) {
    // keep freed blocks in the pool for the next context instead of returning them to the driver
    int dev = 0;
    cudaMemPool_t pool;
    if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
      uint64_t thr = ~0ull;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    pool_ready = true;
  }
  if (cudaStreamCreateWithFlags(&c->up, cudaStreamNonBlocking) != cudaSuccess)
    return pg_set_err(c, PG_ERR_DEVICE, "allocation stream creation failed");
  return 0;
}

int pg_alloc_sync(pg_ctx* c) {
  if (c->up && cudaStreamSynchronize(c->up) != cudaSuccess) return pg_set_err(c, PG_ERR_DEVICE, "device allocation failed");
  return 0;
}

extern "C" {

static int create_host(const pg_problem_desc* d, pg_ctx** out, bool device_prep, bool device_pattern) {
  if (!d || !out) return PG_ERR_INPUT;
  *out = nullptr;
  pg_ctx* c = new pg_ctx;
  pg::ProblemDesc pd;
  pd.elem_type = d->elem_type;
  for (int i = 0; i < 3; ++i) { pd.n[i] = d->n[i]; pd.lo[i] = d->lo[i]; pd.hi[i] = d->hi[i]; }
  const int dim = (d->elem_type == PG_TET4) ? 3 : 2;
  if (d->n_incl < 0 || (d->n_incl > 0 && !d->incl)) { delete c; return PG_ERR_INPUT; }
  pd.incl.assign(d->incl, d->incl + (size_t)d->n_incl * (dim + 1));
  pd.E_matrix = d->E_matrix; pd.nu_matrix = d->nu_matrix; pd.E_fiber = d->E_fiber; pd.nu_fiber = d->nu_fiber;
  pd.coh_law = d->coh_law;
  for (int i = 0; i < 4; ++i) pd.coh[i] = d->coh[i];
  pd.plane_strain = d->plane_strain; pd.subscale = d->subscale;
  for (int i = 0; i < 6; ++i) pd.eps_macro[i] = d->eps_macro[i];
  pd.app_strain = d->app_strain;
  pd.ply_frac = d->ply_frac;
  for (int i = 0; i < 5; ++i) pd.ply[i] = d->ply[i];
  pg::PrepResult pr;
  if (device_prep) {
    std::string why;
    if (pg::device_prep(pd, pr, why)) { c->err = why; *out = c; return PG_ERR_DEVICE; }
    c->prep_ms = pr.valid ? pr.device_ms : -1.0;
    pr.pattern_on_device = pr.valid && device_pattern;
  }
  int rc = pg::build_setup(pd, c->s, device_prep ? &pr : nullptr);
  if (!rc && pr.pattern_on_device) {
    // the adjacency and the CSR pattern on the device too
    std::string why;
    double ms = 0.0;
    const int r2 = pg::device_pattern(c->s, why, &ms);
    if (r2) { c->err = why; *out = c; return r2 == 10 ? PG_ERR_DEVICE : PG_ERR_INPUT; }
    c->prep_ms += ms;
  }
  if (rc) { c->err = c->s.error; *out = c; return rc == 2 ? PG_ERR_INPUT : (rc == 4 ? PG_ERR_UNSUPPORTED : (rc == 7 ? PG_ERR_JACOBIAN : PG_ERR_GEOMETRY)); }
  c->n_coh_qp = (int)c->s.cqp_wgt.size();
  *out = c;
  return 0;
}

int pg_create_host(const pg_problem_desc* d, pg_ctx** out) { return create_host(d, out, false, false); }

int pg_create_prep_device(const pg_problem_desc* d, int passes, pg_ctx** out) {
  if (!(passes & PG_PREP_NODES)) return create_host(d, out, false, false);
  return create_host(d, out, true, (passes & PG_PREP_PATTERN) != 0);
}

int pg_prep_device_ms(const pg_ctx* c, double* ms) {
  if (!c || !ms) return PG_ERR_INPUT;
  *ms = c->prep_ms;
  return 0;
}

int pg_upload(pg_ctx* c) {
  if (!c) return PG_ERR_INPUT;
  pg::Setup& s = c->s;
  const int dim = s.dim;

  // ---- derived row-ownership tables
  const int n_nodes = s.n_std + s.n_enr;
  std::vector<uint8_t> mask(s.n_dn, 0);
  for (int a = 0; a < s.n_dn; ++a) {
    const int na = s.dn_node[a];
    for (int q = 0; q < dim; ++q) if (s.node_dof[(size_t)na * dim + q] < s.n_free) mask[a] |= (uint8_t)(1 << q);
  }
  // neighbour masks, adjacency slots, fast/general split
  std::vector<uint8_t> nbr_mask(s.dn_nbr.size());
  for (size_t k = 0; k < s.dn_nbr.size(); ++k) nbr_mask[k] = mask[s.dn_nbr[k]];
  std::vector<int> slot32(s.dn_adj.size(), 0), slot_off(s.dn_adj.size() + 1, 0);
  std::vector<uint8_t> slots;
  const int maxnb = (dim == 2) ? 9 : 15;
  std::vector<int> fast, slow;
  int maxnb_general = 1;
  for (int a = 0; a < s.n_dn; ++a) {
    const int* nb = s.dn_nbr.data() + s.dn_nbr_off[a];
    const int nn = s.dn_nbr_off[a + 1] - s.dn_nbr_off[a];
    if (nn > 255) return set_err(c, PG_ERR_UNSUPPORTED, "a DOF node with more than 255 neighbours");
    bool ok = nn <= maxnb;
    for (int k = s.dn_adj_off[a]; k < s.dn_adj_off[a + 1]; ++k) {
      const int e = s.dn_adj[k] >> 5;
      std::vector<int> en;
      if (s.cut_of[e] < 0) { ok = ok && true; for (int q = 0; q < s.npe; ++q) en.push_back(s.conn[(size_t)e * s.npe + q]); }
      else {
        ok = false;
        const int cc = s.cut_of[e];
        for (int q = s.cut_node_off[cc]; q < s.cut_node_off[cc + 1]; ++q) en.push_back(s.cut_nodes[q]);
      }
      slot_off[k] = (int)slots.size();
      const size_t first_slot = slots.size();
      for (size_t lb = 0; lb < en.size(); ++lb) {
        const int db = s.node_dn[en[lb]];
        const int pos = (int)(std::lower_bound(nb, nb + nn, db) - nb);
        if (pos >= nn || nb[pos] != db) return set_err(c, PG_ERR_STATE, "internal: adjacency without neighbour slot");
        // the lanes of a row group add an element's blocks concurrently: its nodes need distinct slots
        for (size_t k2 = first_slot; k2 < slots.size(); ++k2)
          if (slots[k2] == pos) return set_err(c, PG_ERR_UNSUPPORTED, "an element holds a node and its periodic image");
        slots.push_back((uint8_t)pos);
        if (s.cut_of[e] < 0) slot32[k] |= pos << (8 * lb);
      }
    }
    slot_off[s.dn_adj.size()] = (int)slots.size();
    (void)ok;
    slow.push_back(a);
    maxnb_general = std::max(maxnb_general, nn);
  }
  slot_off[s.dn_adj.size()] = (int)slots.size();
  // Structured-grid stencil nodes (pg_stencil.cuh): interior DOF nodes two cells from the domain
  // boundary whose adjacency, neighbours and row layout match their class table exactly, whose
  // elements are all uncut and whose neighbour DOFs are all free.  Everything else is general.
  std::vector<int4> stencil;
  {
    const int Nx = s.desc.n[0], Ny = s.desc.n[1], Nz = (dim == 3) ? s.desc.n[2] : 0;
    const int sx = Nx + 1, sxy = sx * (Ny + 1);
    const bool grid_ok = (s.etype == pg::TRI3 || s.etype == pg::TET4);
    std::vector<char> in_stencil(s.n_dn, 0);
    std::vector<std::vector<int4>> by_class(2);
    for (int a = 0; a < s.n_dn && grid_ok; ++a) {
      const int nid = s.dn_node[a];
      if (nid >= s.n_std) continue;
      const int i = nid % sx, j = (nid / sx) % (Ny + 1), k = nid / sxy;
      if (i < 2 || i > Nx - 2 || j < 2 || j > Ny - 2) continue;
      if (dim == 3 && (k < 2 || k > Nz - 2)) continue;
      const int cls = (dim == 2) ? ((i + j) % 2) : 0;
      const int NN = (dim == 2) ? (cls == 0 ? pgd::Tri3Stencil0::NN : pgd::Tri3Stencil1::NN) : pgd::Tet4Stencil0::NN;
      const int NADJ = (dim == 2) ? (cls == 0 ? pgd::Tri3Stencil0::NADJ : pgd::Tri3Stencil1::NADJ) : pgd::Tet4Stencil0::NADJ;
      auto off = [&](int q, int d) {
        return (dim == 2) ? (cls == 0 ? pgd::Tri3Stencil0::off(q, d) : pgd::Tri3Stencil1::off(q, d)) : pgd::Tet4Stencil0::off(q, d);
      };
      auto entv = [&](int q, int cidx) {
        return (dim == 2) ? (cls == 0 ? pgd::Tri3Stencil0::ent(q, cidx) : pgd::Tri3Stencil1::ent(q, cidx)) : pgd::Tet4Stencil0::ent(q, cidx);
      };
      bool ok = (s.dn_nbr_off[a + 1] - s.dn_nbr_off[a]) == NN && (s.dn_adj_off[a + 1] - s.dn_adj_off[a]) == NADJ;
      for (int q = 0; ok && q < NN; ++q) {
        const int nb = s.dn_node[s.dn_nbr[s.dn_nbr_off[a] + q]];
        ok = nb == nid + off(q, 0) + off(q, 1) * sx + off(q, 2) * sxy && mask[s.dn_nbr[s.dn_nbr_off[a] + q]] == (1 << dim) - 1;
      }
      for (int q = 0; ok && q < NADJ; ++q) {
        const int ci = i + entv(q, 0), cj = j + entv(q, 1), ck = k + entv(q, 2);
        const int e = (dim == 2) ? 2 * (cj * Nx + ci) + entv(q, 3) : 6 * ((ck * Ny + cj) * Nx + ci) + entv(q, 3);
        const int entry = s.dn_adj[s.dn_adj_off[a] + q];
        ok = (entry >> 5) == e && (entry & 31) == entv(q, 4) && s.cut_of[e] < 0;
        for (int n = 0; ok && n <= dim; ++n) {
          const int sl = entv(q, 5 + n);
          ok = s.conn[(size_t)e * (dim + 1) + n] == nid + off(sl, 0) + off(sl, 1) * sx + off(sl, 2) * sxy;
        }
      }
      if (!ok) continue;
      const int g0 = s.node_dof[(size_t)nid * dim];
      for (int q = 0; ok && q < dim; ++q) ok = s.node_dof[(size_t)nid * dim + q] == g0 + q && g0 + q < s.n_free;
      if (!ok) continue;
      const int row0 = s.rp[0][g0];
      for (int q = 0; ok && q < dim; ++q)
        ok = s.rp[0][g0 + q] == row0 + q * NN * dim && s.rp[0][g0 + q + 1] - s.rp[0][g0 + q] == NN * dim &&
             s.rp[1][g0 + q + 1] == s.rp[1][g0 + q];
      if (!ok) continue;
      by_class[cls].push_back(make_int4(nid, g0, row0, cls));
      in_stencil[a] = 1;
    }
    // each class segment padded to whole warps (entries with node -1): a warp's nodes then share
    // one class and one row length, which the staged row stores of the 2D kernel rely on
    for (int cls = 0; cls < 2; ++cls) {
      auto& v = by_class[cls];
      if (v.empty()) continue;
      stencil.insert(stencil.end(), v.begin(), v.end());
      while (stencil.size() % 32) stencil.push_back(make_int4(-1, 0, 0, cls));
    }
    // 2D tiles of 16 x 8 grid nodes (pg_tile.cuh): per tile 64 class-0 then 64 class-1 node
    // entries in row-major order, each with its run's offset in the tile's stage (a tile row of
    // nodes is 8 runs of 36 and 8 of 20 values), and the contiguous CSR segments of each tile row
    if (dim == 2 && grid_ok) {
      std::vector<int4> st_of(s.n_std, make_int4(-1, 0, 0, 0));
      for (int cls = 0; cls < 2; ++cls)
        for (const int4& v : by_class[cls]) st_of[v.x] = v;
      const int runlen[2] = {2 * pgd::Tri3Stencil0::NN * 2, 2 * pgd::Tri3Stencil1::NN * 2};
      std::vector<int4> tiles, tnodes, segs;
      for (int j0 = 0; j0 <= Ny; j0 += pgd::kTileY)
        for (int i0 = 0; i0 <= Nx; i0 += pgd::kTileX) {
          std::vector<int4> ent[2];
          std::vector<int4> tsg;
          bool any = false;
          for (int r = 0; r < pgd::kTileY; ++r) {
            int off = r * pgd::kTileRowStage;
            int4 seg = make_int4(-1, 0, 0, 0);
            int seg_next = -1;   // CSR slot that continues the open segment
            for (int cc = 0; cc < pgd::kTileX; ++cc) {
              const int i = i0 + cc, j = j0 + r;
              const int cls = (i + j) % 2;
              int4 e = make_int4(-1, 0, 0, 0);
              if (i <= Nx && j <= Ny && st_of[j * sx + i].x >= 0) {
                const int4 v = st_of[j * sx + i];
                e = make_int4(v.x, v.y, v.z, off);
                any = true;
                if (seg.x >= 0 && v.z == seg_next) {
                  seg.z += runlen[cls];
                } else {
                  if (seg.x >= 0) tsg.push_back(seg);
                  seg = make_int4(off, v.z, runlen[cls], 0);
                }
                seg_next = v.z + runlen[cls];
              } else if (seg.x >= 0) {
                tsg.push_back(seg);
                seg = make_int4(-1, 0, 0, 0);
              }
              ent[cls].push_back(e);
              off += runlen[cls];
            }
            if (seg.x >= 0) tsg.push_back(seg);
          }
          if (!any) continue;
          if (ent[0].size() != 64 || ent[1].size() != 64) return set_err(c, PG_ERR_STATE, "internal: tile classes");
          tiles.push_back(make_int4(i0, j0, (int)segs.size(), (int)tsg.size()));
          tnodes.insert(tnodes.end(), ent[0].begin(), ent[0].end());
          tnodes.insert(tnodes.end(), ent[1].begin(), ent[1].end());
          segs.insert(segs.end(), tsg.begin(), tsg.end());
        }
      PG_TRY(upload(c, tiles, &c->tiles));
      PG_TRY(upload(c, tnodes, &c->tnodes));
      PG_TRY(upload(c, segs, &c->tsegs));
      c->n_tiles = (int)tiles.size();
    }
    // 3D tiles of 4 x 4 x 4 grid nodes (pg_tile.cuh): per tile {i0, j0, k0, 0} and {first
    // segment, segments, 0, 0}; 64 node entries (x fastest) with their run's stage offset (a
    // node's three rows are one run of 135 values); the contiguous CSR segments of each x-row
    if (dim == 3 && grid_ok) {
      std::vector<int4> st_of(s.n_std, make_int4(-1, 0, 0, 0));
      for (const int4& v : by_class[0]) st_of[v.x] = v;
      constexpr int T3 = pgd::kT3, RUN = pgd::kT3Run;
      std::vector<int4> tiles, tnodes, segs;
      for (int k0 = 0; k0 <= Nz; k0 += T3)
        for (int j0 = 0; j0 <= Ny; j0 += T3)
          for (int i0 = 0; i0 <= Nx; i0 += T3) {
            std::vector<int4> ent, tsg;
            bool any = false;
            for (int lk = 0; lk < T3; ++lk)
              for (int lj = 0; lj < T3; ++lj) {
                int4 seg = make_int4(-1, 0, 0, 0);
                int seg_next = -1;
                for (int li = 0; li < T3; ++li) {
                  const int i = i0 + li, j = j0 + lj, k = k0 + lk;
                  const int off = ((lk * T3 + lj) * T3 + li) * RUN;
                  int4 e = make_int4(-1, 0, 0, 0);
                  if (i <= Nx && j <= Ny && k <= Nz && st_of[k * sxy + j * sx + i].x >= 0) {
                    const int4 v = st_of[k * sxy + j * sx + i];
                    e = make_int4(v.x, v.y, v.z, off);
                    any = true;
                    if (seg.x >= 0 && v.z == seg_next) seg.z += RUN;
                    else {
                      if (seg.x >= 0) tsg.push_back(seg);
                      seg = make_int4(off, v.z, RUN, 0);
                    }
                    seg_next = v.z + RUN;
                  } else if (seg.x >= 0) {
                    tsg.push_back(seg);
                    seg = make_int4(-1, 0, 0, 0);
                  }
                  ent.push_back(e);
                }
                if (seg.x >= 0) tsg.push_back(seg);
              }
            if (!any) continue;
            tiles.push_back(make_int4(i0, j0, k0, 0));
            tiles.push_back(make_int4((int)segs.size(), (int)tsg.size(), 0, 0));
            tnodes.insert(tnodes.end(), ent.begin(), ent.end());
            segs.insert(segs.end(), tsg.begin(), tsg.end());
          }
      PG_TRY(upload(c, tiles, &c->tiles));
      PG_TRY(upload(c, tnodes, &c->tnodes));
      PG_TRY(upload(c, segs, &c->tsegs));
      c->n_tiles = (int)tiles.size() / 2;
    }
    std::vector<int> rest;
    maxnb_general = 1;
    for (int a = 0; a < s.n_dn; ++a)
      if (!in_stencil[a]) { rest.push_back(a); maxnb_general = std::max(maxnb_general, s.dn_nbr_off[a + 1] - s.dn_nbr_off[a]); }
    // general nodes grouped by shape (cut adjacent elements, then all adjacent elements, both
    // descending; node order within a group) so the lane groups of a warp walk alike entries
    auto n_cut_adj = [&](int a) {
      int k = 0;
      for (int j = s.dn_adj_off[a]; j < s.dn_adj_off[a + 1]; ++j) k += s.cut_of[s.dn_adj[j] >> 5] >= 0;
      return k;
    };
    std::stable_sort(rest.begin(), rest.end(), [&](int x, int y) {
      const int cx = n_cut_adj(x), cy = n_cut_adj(y);
      if (cx != cy) return cx > cy;
      return (s.dn_adj_off[x + 1] - s.dn_adj_off[x]) > (s.dn_adj_off[y + 1] - s.dn_adj_off[y]);
    });
    slow.swap(rest);
    fast.clear();
    for (auto& v : stencil) if (v.x >= 0) fast.push_back(s.node_dn[v.x]);
    c->grid = pgd::GridInfo{Nx, Ny, Nz};
  }
  // cut-element scratch layout
  std::vector<long long> ke_off(s.ncut + 1, 0);
  std::vector<int> re_off(s.ncut + 1, 0);
  for (int cc = 0; cc < s.ncut; ++cc) {
    const int nd = (s.cut_node_off[cc + 1] - s.cut_node_off[cc]) * dim;
    c->max_nd = std::max(c->max_nd, nd);
    ke_off[cc + 1] = ke_off[cc] + (long long)nd * nd;
    re_off[cc + 1] = re_off[cc] + nd;
  }
  c->cut_scratch = ke_off[s.ncut];
  c->n_coh_qp = (int)s.cqp_wgt.size();

  // descriptors of the general rows (k_rows_general)
  std::vector<int4> gdesc, adesc;
  std::vector<int> growd;
  std::vector<int4> aresd;   // per entry: uncut {element nodes}, cut {cut element, first node, cohesive place, 0}
  for (int a : slow) {
    const int na = s.dn_node[a];
    gdesc.push_back(make_int4((int)adesc.size(), s.dn_adj_off[a + 1] - s.dn_adj_off[a], s.dn_nbr_off[a],
                              s.dn_nbr_off[a + 1] - s.dn_nbr_off[a]));
    int rows[3][3];
    for (int q = 0; q < dim; ++q) {
      const int gq = s.node_dof[(size_t)na * dim + q];
      const bool rf = gq < s.n_free;
      const int rr = rf ? gq : gq - s.n_free;
      rows[0][q] = gq;
      rows[1][q] = rf ? s.rp[0][rr] : s.rp[2][rr];
      rows[2][q] = rf ? s.rp[1][rr] : s.rp[3][rr];
    }
    for (int t = 0; t < 3; ++t) for (int q = 0; q < dim; ++q) growd.push_back(rows[t][q]);
    // cut elements first, then uncut ones, each in adjacency order
    for (int pass = 0; pass < 2; ++pass)
    for (int k = s.dn_adj_off[a]; k < s.dn_adj_off[a + 1]; ++k) {
      const int e = s.dn_adj[k] >> 5, la = s.dn_adj[k] & 31;
      const int cc = s.cut_of[e];
      if ((cc >= 0) != (pass == 0)) continue;
      if (cc < 0) {
        adesc.push_back(make_int4(e, la, slot32[k], s.elem_mat[e]));
        const int* en = &s.conn[(size_t)e * s.npe];
        aresd.push_back(make_int4(en[0], en[1], en[2], s.npe > 3 ? en[3] : -1));
      } else {
        const int mn = s.cut_node_off[cc + 1] - s.cut_node_off[cc];
        adesc.push_back(make_int4(e, la | (mn << 8), slot_off[k], 0));
        // the row node's place on a cohesive element of this cut element: (element << 5 | position)
        int cpa = -1;
        for (int ce = s.cut_coh_off[cc]; ce < s.cut_coh_off[cc + 1] && cpa < 0; ++ce)
          for (int j = s.coh_local_off[ce]; j < s.coh_local_off[ce + 1]; ++j)
            if (s.coh_local[j] == la) { cpa = ce * 32 + (j - s.coh_local_off[ce]); break; }
        aresd.push_back(make_int4(cc, s.cut_node_off[cc], cpa, 0));
      }
    }
    // k_rows_general walks a node's cut entries until the first uncut one: every node's entries
    // must be cut-first
    for (size_t k = (size_t)gdesc.back().x + 1; k < adesc.size(); ++k)
      if ((adesc[k].y >> 8) != 0 && (adesc[k - 1].y >> 8) == 0)
        return set_err(c, PG_ERR_STATE, "internal: a cut entry after an uncut one in a general row");
  }

  // ---- device residency
  pgd::DevProblem& P = c->P;
  P.dim = dim; P.npe = s.npe; P.nvoigt = s.nvoigt;
  P.n_nodes = n_nodes; P.ne = s.ne; P.ncut = s.ncut; P.n_dn = s.n_dn;
  P.n_free = s.n_free; P.n_const = s.n_const; P.subscale = s.desc.subscale;
  for (int m = 0; m < 3; ++m) for (int i = 0; i < 36; ++i) { P.D[m][i] = s.D[m][i]; P.Df[m][i] = (float)s.D[m][i]; }
  P.coh.law = s.coh.law; P.coh.nvar = s.coh.nvar; P.coh.sigma_c = s.coh.sigma_c; P.coh.delta_c1 = s.coh.delta_c1;
  P.coh.delta_c2 = s.coh.delta_c2; P.coh.delta_cn = s.coh.delta_cn; P.coh.delta_ct = s.coh.delta_ct; P.coh.q = s.coh.q;
  P.coh.delta_c = s.coh.delta_c; P.coh.beta2 = s.coh.beta2; P.coh.alpha = s.coh.alpha; P.coh.delta_c3 = s.coh.delta_c3;
  {
    std::vector<double> Dh(108);
    std::vector<float> Dfh(108);
    for (int m = 0; m < 3; ++m) for (int i = 0; i < 36; ++i) { Dh[m * 36 + i] = s.D[m][i]; Dfh[m * 36 + i] = (float)s.D[m][i]; }
    PG_TRY(upload(c, Dh, &P.Dd));
    PG_TRY(upload(c, Dfh, &P.Dfd));
  }
  if ((dim == 2 ? pgl::tile_consts<2>(c, P) : pgl::tile_consts<3>(c, P)) != 0)
    return set_err(c, PG_ERR_DEVICE, "tile shape constants failed");
  std::vector<float> Xf(s.X.begin(), s.X.end());
  PG_TRY(upload(c, s.X, &P.X));
  PG_TRY(upload(c, Xf, &P.Xf));
  PG_TRY(upload(c, s.conn, &P.conn));
  PG_TRY(upload(c, s.elem_mat, &P.emat));
  PG_TRY(upload(c, s.cut_of, &P.cut_of));
  PG_TRY(upload(c, s.node_dof, &P.node_dof));
  PG_TRY(upload(c, s.node_dn, &P.node_dn));
  PG_TRY(upload(c, s.cut_node_off, &P.cut_node_off));
  PG_TRY(upload(c, s.cut_nodes, &P.cut_nodes));
  // Device quadrature tables: the quadrature points of an affine (tri3 / tet4) sub-element of an
  // affine parent share one gradient set, so they are merged into one point carrying the sum of
  // their weights (w_0 + w_1 + ... in rule order).  K and R change only by rounding.
  {
    std::vector<int> dq_off(1, 0), dq_mat, dg_off(1, 0);
    std::vector<double> dq_w, dg;
    for (int cc = 0; cc < s.ncut; ++cc) {
      int qp = s.cut_qp_off[cc];
      for (int sb = s.cut_sub_off[cc]; sb < s.cut_sub_off[cc + 1]; ++sb) {
        const int st = s.sub_type[sb];
        const int nq = s.sub_qp_off[sb + 1] - s.sub_qp_off[sb];
        if (s.sub_qp_off[sb] != qp) return set_err(c, PG_ERR_STATE, "internal: quadrature offsets out of order");
        // (a quad4 parent's gradients vary from point to point, so its sub-elements never merge)
        const bool affine = (st == pg::SUB_TRI3 || st == pg::SUB_TET4) && s.etype != pg::QUAD4;
        if (affine) {
          double w = 0.0;
          for (int q = 0; q < nq; ++q) w += s.qp_wgt[qp + q];
          dq_w.push_back(w);
          dq_mat.push_back(s.qp_mat[qp]);
          dg.insert(dg.end(), s.qp_grad.begin() + s.qp_grad_off[qp], s.qp_grad.begin() + s.qp_grad_off[qp + 1]);
          dg_off.push_back((int)dg.size());
        } else {
          for (int q = 0; q < nq; ++q) {
            dq_w.push_back(s.qp_wgt[qp + q]);
            dq_mat.push_back(s.qp_mat[qp + q]);
            dg.insert(dg.end(), s.qp_grad.begin() + s.qp_grad_off[qp + q], s.qp_grad.begin() + s.qp_grad_off[qp + q + 1]);
            dg_off.push_back((int)dg.size());
          }
        }
        qp += nq;
      }
      if (qp != s.cut_qp_off[cc + 1]) return set_err(c, PG_ERR_STATE, "internal: quadrature count mismatch");
      dq_off.push_back((int)dq_w.size());
    }
    for (int cc = 0; cc < s.ncut; ++cc) {
      c->max_cut_qp = std::max(c->max_cut_qp, dq_off[cc + 1] - dq_off[cc]);
      c->max_cut_nodes = std::max(c->max_cut_nodes, s.cut_node_off[cc + 1] - s.cut_node_off[cc]);
    }
    {
      // size classes: at most 8 points and 8 nodes (one fiber: tri3 + quad4 sub-elements), the rest
      std::vector<int> lists[2];
      for (int cc = 0; cc < s.ncut; ++cc) {
        const int nq = dq_off[cc + 1] - dq_off[cc], mn = s.cut_node_off[cc + 1] - s.cut_node_off[cc];
        const int cls = (nq <= 8 && mn <= 8) ? 0 : 1;
        lists[cls].push_back(cc);
        c->cut_cls_qp[cls] = std::max(c->cut_cls_qp[cls], nq);
        c->cut_cls_nodes[cls] = std::max(c->cut_cls_nodes[cls], mn);
      }
      for (int cls = 0; cls < 2; ++cls) {
        PG_TRY(upload(c, lists[cls], &c->cut_list[cls]));
        c->n_cut_list[cls] = (int)lists[cls].size();
      }
    }
    PG_TRY(upload(c, dq_off, &P.cut_qp_off));
    PG_TRY(upload(c, dq_w, &P.qp_wgt));
    PG_TRY(upload(c, dq_mat, &P.qp_mat));
    PG_TRY(upload(c, dg_off, &P.qp_grad_off));
    PG_TRY(upload(c, dg, &P.qp_grad));
  }
  PG_TRY(upload(c, s.cut_coh_off, &P.cut_coh_off));
  PG_TRY(upload(c, s.coh_nh, &P.coh_nh));
  PG_TRY(upload(c, s.coh_local_off, &P.coh_local_off));
  PG_TRY(upload(c, s.coh_local, &P.coh_local));
  PG_TRY(upload(c, s.coh_qp_off, &P.coh_qp_off));
  PG_TRY(upload(c, s.cqp_N, &P.cqp_N));
  {
    std::vector<int> noff;
    noff.reserve(s.cqp_wgt.size() + 1);
    for (size_t ce = 0; ce + 1 < s.coh_qp_off.size(); ++ce)
      for (int cq = s.coh_qp_off[ce]; cq < s.coh_qp_off[ce + 1]; ++cq) noff.push_back(0);
    // running offsets: each point of cohesive element ce holds coh_nh[ce] shape values
    int o = 0, k = 0;
    for (size_t ce = 0; ce + 1 < s.coh_qp_off.size(); ++ce)
      for (int cq = s.coh_qp_off[ce]; cq < s.coh_qp_off[ce + 1]; ++cq) { noff[k++] = o; o += s.coh_nh[ce]; }
    if (o != (int)s.cqp_N.size()) return set_err(c, PG_ERR_STATE, "internal: cohesive shape-value count mismatch");
    PG_TRY(upload(c, noff, &P.cqp_noff));
  }
  PG_TRY(upload(c, s.cqp_R, &P.cqp_R));
  PG_TRY(upload(c, s.cqp_wgt, &P.cqp_wgt));
  PG_TRY(upload(c, s.cqp_isv, &P.cqp_isv));
  PG_TRY(upload(c, ke_off, &P.ke_off));
  PG_TRY(upload(c, re_off, &P.re_off));
  // the cut elements' volumetric blocks: set-up only (reduced into the static rows, then released)
  double* dke = nullptr;
  PG_TRY(dalloc(c, (size_t)ke_off[s.ncut], &dke));
  P.ke = dke;
  PG_TRY(dalloc(c, (size_t)s.n_isv, &c->d_isv_committed));
  PG_TRY(dalloc(c, (size_t)s.n_isv, &c->d_isv_trial));
  P.isv_committed = c->d_isv_committed; P.isv_trial = c->d_isv_trial;
  PG_TRY(dalloc(c, (size_t)c->n_coh_qp, &c->d_zone));
  P.zone = c->d_zone;
  PG_TRY(upload(c, s.dn_node, &P.dn_node));
  PG_TRY(upload(c, s.dn_nbr_off, &P.dn_nbr_off));
  PG_TRY(upload(c, nbr_mask, &P.dn_nbr_mask));
  PG_TRY(upload(c, s.dn_adj_off, &P.dn_adj_off));
  PG_TRY(upload(c, s.dn_adj, &P.dn_adj));
  PG_TRY(upload(c, slot32, &P.adj_slot32));
  PG_TRY(upload(c, slot_off, &P.adj_slot_off));
  PG_TRY(upload(c, slots, &P.adj_slots));
  PG_TRY(upload(c, fast, &P.fast_dn));
  PG_TRY(upload(c, slow, &P.slow_dn));
  {
    const int4* dst = nullptr;
    PG_TRY(upload(c, stencil, &dst));
    c->stencil = dst;
    c->n_stencil = (int)stencil.size();
  }
  c->fast_dn = fast;
  c->slow_dn = slow;

  P.n_fast_dn = (int)fast.size(); P.n_slow_dn = (int)slow.size();
  P.maxnb_general = maxnb_general;
  PG_TRY(upload(c, gdesc, &P.gdesc));
  PG_TRY(upload(c, growd, &P.growd));
  PG_TRY(upload(c, adesc, &P.adesc));
  PG_TRY(upload(c, aresd, &P.aresd));
  // cohesive elements: owning cut element, scratch offsets of their blocks, and the cohesive
  // position of every cut-element local node (a node is on at most one cohesive element)
  std::vector<int> kc_off_h, cohpos_h;
  {
    const int n_ce = (int)s.coh_nh.size();
    if ((long long)n_ce * 32 > 2147483647LL) return set_err(c, PG_ERR_UNSUPPORTED, "too many cohesive elements");
    std::vector<int> ce_cut(n_ce), kc_off(n_ce + 1, 0), cohpos(s.cut_nodes.size(), -1);
    for (int cc = 0; cc < s.ncut; ++cc)
      for (int ce = s.cut_coh_off[cc]; ce < s.cut_coh_off[cc + 1]; ++ce) {
        ce_cut[ce] = cc;
        const int nh = s.coh_nh[ce];
        if (2 * nh > 32) return set_err(c, PG_ERR_UNSUPPORTED, "cohesive element with more than 32 nodes");
        kc_off[ce + 1] = kc_off[ce] + nh * nh * dim * dim + nh * dim;
        for (int k = 0; k < 2 * nh; ++k) {
          const int ln = s.coh_local[s.coh_local_off[ce] + k];
          int& slot = cohpos[s.cut_node_off[cc] + ln];
          if (slot >= 0) return set_err(c, PG_ERR_STATE, "internal: a node on two cohesive elements of one cut element");
          slot = ce * 32 + k;
        }
      }
    PG_TRY(upload(c, ce_cut, &P.ce_cut));
    {
      // node ids of the cohesive elements' local nodes, laid out like coh_local
      std::vector<int> gnode(s.coh_local.size());
      for (int ce = 0; ce < n_ce; ++ce)
        for (int k = s.coh_local_off[ce]; k < s.coh_local_off[ce + 1]; ++k)
          gnode[k] = s.cut_nodes[s.cut_node_off[ce_cut[ce]] + s.coh_local[k]];
      PG_TRY(upload(c, gnode, &P.coh_gnode));
    }
    PG_TRY(upload(c, kc_off, &P.kc_off));
    PG_TRY(upload(c, cohpos, &P.cohpos));
    kc_off_h = kc_off;
    cohpos_h = cohpos;
    double* dk;
    PG_TRY(dalloc(c, (size_t)kc_off[n_ce], &dk));
    P.kcoh = dk;
    P.n_coh_el = n_ce;
    P.n_coh_qp = c->n_coh_qp;
    int max_mn = 1;
    for (int cc = 0; cc < s.ncut; ++cc) max_mn = std::max(max_mn, s.cut_node_off[cc + 1] - s.cut_node_off[cc]);
    P.max_mn = max_mn;
  }
  // row positions: free DOFs of the earlier neighbours of every neighbour slot
  {
    std::vector<int> pre(s.dn_nbr.size(), 0);
    for (int a = 0; a < s.n_dn; ++a) {
      int acc = 0;
      for (int k = s.dn_nbr_off[a]; k < s.dn_nbr_off[a + 1]; ++k) { pre[k] = acc; acc += __builtin_popcount(nbr_mask[k]); }
    }
    PG_TRY(upload(c, pre, &P.nbr_pre));
  }
  // side: the structured tiles at the lowest priority; side2: the general chain at the highest
  {
    int least = 0, greatest = 0;
    if (cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess ||
        cudaStreamCreateWithPriority(&c->side, cudaStreamNonBlocking, least) != cudaSuccess ||
        cudaStreamCreateWithPriority(&c->side2, cudaStreamNonBlocking, greatest) != cudaSuccess)
      return set_err(c, PG_ERR_DEVICE, "stream creation failed");
  }
  for (int b = 0; b < 4; ++b) {
    PG_TRY(upload(c, s.rp[b], &P.rp[b]));
    PG_TRY(dalloc(c, s.ci[b].size(), &P.val[b]));
  }
  // The values a later assembly can change (PG_KEEP_STATIC, pg_changing_values): every bulk law
  // is linear elastic, so only the entries coupling DOFs of nodes on one cohesive element depend
  // on the state; each block's changing values lie in the rows from the smallest such DOF on.
  {
    int fmin = s.n_free, pmin = s.n_const;
    for (int cc = 0; cc < s.ncut; ++cc)
      for (int ce = s.cut_coh_off[cc]; ce < s.cut_coh_off[cc + 1]; ++ce)
        for (int q = s.coh_local_off[ce]; q < s.coh_local_off[ce + 1]; ++q) {
          const int node = s.cut_nodes[s.cut_node_off[cc] + s.coh_local[q]];
          for (int d = 0; d < dim; ++d) {
            const int dof = s.node_dof[(size_t)node * dim + d];
            if (dof < s.n_free) fmin = std::min(fmin, dof);
            else pmin = std::min(pmin, dof - s.n_free);
          }
        }
    const bool fr = fmin < s.n_free, pr = pmin < s.n_const;
    long long nnz[4];
    for (int b = 0; b < 4; ++b) nnz[b] = (long long)s.ci[b].size();
    c->changing_from[0] = fr ? s.rp[0][fmin] : nnz[0];
    c->changing_from[1] = (fr && pr) ? s.rp[1][fmin] : nnz[1];
    c->changing_from[2] = (fr && pr) ? s.rp[2][pmin] : nnz[2];
    c->changing_from[3] = pr ? s.rp[3][pmin] : nnz[3];
    c->kept_valid = false;
  }
  PG_TRY(dalloc(c, (size_t)s.n_free, &P.Pf));
  PG_TRY(dalloc(c, (size_t)s.n_const, &P.Pp));
  PG_TRY(dalloc(c, (size_t)n_nodes * dim, &c->d_U));
  PG_TRY(dalloc(c, 1, &c->d_err));
  P.err = c->d_err;
  PG_TRY(dalloc(c, 1024, &c->d_red));
  // Static part of the general rows.  tri3 / tet4: every general node gets one, holding its cut
  // and uncut elements' volumetric blocks (every bulk law is linear elastic, so these do not
  // depend on the state; k_general_static forms them once), and an assembly adds only the
  // cohesive blocks.  quad4: only the general nodes with cut adjacent elements, sorted first, so
  // they form the prefix [0, n_stat).  Each gets its neighbour slots' blocks (slab layout), the
  // slot node ids and a macroscale-strain response.
  {
    const int nv = (dim == 2) ? 3 : 6;
    const bool full_static = s.etype != pg::QUAD4;
    int n_stat = 0;
    for (size_t i = 0; i < slow.size(); ++i) {
      const int4 gd = gdesc[i];
      const bool has_cut = gd.y > 0 && (adesc[gd.x].y >> 8) != 0;   // entries are cut-first
      if (has_cut && (int)i != n_stat) return set_err(c, PG_ERR_STATE, "internal: general nodes next to cut elements are not a prefix");
      if (has_cut) ++n_stat;
    }
    if (full_static) n_stat = (int)slow.size();
    std::vector<int> stat_off(n_stat + 1, 0), stat_node;
    for (int i = 0; i < n_stat; ++i) {
      const int4 gd = gdesc[i];
      stat_off[i + 1] = stat_off[i] + gd.w;
      for (int k = gd.z; k < gd.z + gd.w; ++k) stat_node.push_back(s.dn_node[s.dn_nbr[k]]);
    }
    P.n_stat = n_stat;
    PG_TRY(upload(c, stat_off, &P.stat_slot_off));
    PG_TRY(upload(c, stat_node, &P.stat_node));
    double* dst = nullptr;
    double* dsg = nullptr;
    PG_TRY(dalloc(c, (size_t)stat_off[n_stat] * dim * dim, &dst));
    PG_TRY(dalloc(c, (size_t)n_stat * dim * nv, &dsg));
    P.stat = dst;
    P.stat_g = dsg;
    // Block-parallel general rows (pg_general.cuh; tri3 / tet4): one block per (general node,
    // neighbour slot) with its static index and its cohesive contributions in adjacency order,
    // and per node the traction list (the uncut elements are in the static image)
    if (s.etype != pg::QUAD4) {
      const int D2 = dim * dim;
      std::vector<int4> gblk;
      std::vector<int> gblk_cl(1, 0), gcl, tl_off(1, 0), tl;
      std::vector<std::vector<int>> bcl;
      for (size_t i = 0; i < slow.size(); ++i) {
        const int4 gd = gdesc[i];
        bcl.assign(gd.w, std::vector<int>());
        for (int k = gd.x; k < gd.x + gd.y; ++k) {
          const int4 ad = adesc[k], ax = aresd[k];
          const int mn = ad.y >> 8;
          if (mn == 0) continue;   // uncut: in the static image
          const int cpa = ax.z;
          if (cpa < 0) continue;
          const int ce = cpa >> 5, n1 = cpa & 31, nh = s.coh_nh[ce];
          for (int b = 0; b < mn; ++b) {
            const int cpb = cohpos_h[ax.y + b];
            if (cpb < 0 || (cpb >> 5) != ce) continue;
            const int n2 = cpb & 31;
            const int off = kc_off_h[ce] + ((n1 % nh) * nh + (n2 % nh)) * D2;
            const int neg = ((n1 >= nh) == (n2 >= nh)) ? 0 : 1;
            bcl[slots[ad.z + b]].push_back(off * 2 + neg);
          }
          const int toff = kc_off_h[ce] + nh * nh * D2 + (n1 % nh) * dim;
          tl.push_back(toff * 2 + ((n1 >= nh) ? 0 : 1));
        }
        for (int k = 0; k < gd.w; ++k) {
          gblk.push_back(make_int4((int)i, k, stat_off[i] + k, 0));
          gcl.insert(gcl.end(), bcl[k].begin(), bcl[k].end());
          gblk_cl.push_back((int)gcl.size());
        }
        tl_off.push_back((int)tl.size());
      }
      P.n_gblk = (int)gblk.size();
      PG_TRY(upload(c, gblk, &P.gblk));
      PG_TRY(upload(c, gblk_cl, &P.gblk_cl));
      PG_TRY(upload(c, gcl, &P.gcl));
      PG_TRY(upload(c, tl_off, &P.gnode_tl_off));
      PG_TRY(upload(c, tl, &P.gnode_tl));
    }
    c->stat_doubles = (long long)stat_off[n_stat] * dim * dim + (long long)n_stat * dim * nv;
    if (s.ncut > 0) {
      double* dg = nullptr;
      PG_TRY(dalloc(c, (size_t)re_off[s.ncut] / dim * dim * nv, &dg));
      P.gmac = dg;
      if (dim == 2) { pgl::cut_volumetric<2>(c, P, dg); pgl::general_static<2>(c, P, dst, dsg); }
      else { pgl::cut_volumetric<3>(c, P, dg); pgl::general_static<3>(c, P, dst, dsg); }
      int herr = 0;
      cudaMemcpyAsync(&herr, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->up);
      if (cudaStreamSynchronize(c->up) != cudaSuccess) return set_err(c, PG_ERR_DEVICE, "cut-element set-up kernel failed");
      if (herr) return set_err(c, PG_ERR_NONFINITE, "non-finite cut-element stiffness at set-up");
      // the per-element blocks are reduced: give their memory back
      for (double* p : {dke, dg}) pg_untrack_free(c, p);
      P.ke = nullptr;
      P.gmac = nullptr;
    } else if (full_static && n_stat > 0) {
      // no cut elements: the image holds the uncut elements alone
      if (dim == 2) pgl::general_static<2>(c, P, dst, dsg);
      else pgl::general_static<3>(c, P, dst, dsg);
      int herr = 0;
      cudaMemcpyAsync(&herr, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->up);
      if (cudaStreamSynchronize(c->up) != cudaSuccess) return set_err(c, PG_ERR_DEVICE, "general-row set-up kernel failed");
      if (herr) return set_err(c, PG_ERR_NONFINITE, "non-finite general-row stiffness at set-up");
    }
  }
  return pg_alloc_sync(c);
}

int pg_create(const pg_problem_desc* d, pg_ctx** out) {
  int rc = pg_create_host(d, out);
  if (rc) return rc;
  return pg_upload(*out);
}

int pg_debug_array(const pg_ctx* c, const char* name, int64_t* n, const void** ptr) {
  if (!c || !name || !n || !ptr) return 0;
  const pg::Setup& s = c->s;
  struct { const char* k; const void* p; size_t n; int kind; } tab[] = {
      {"cut_elem", s.cut_elem.data(), s.cut_elem.size(), 1}, {"cut_node_off", s.cut_node_off.data(), s.cut_node_off.size(), 1},
      {"cut_nodes", s.cut_nodes.data(), s.cut_nodes.size(), 1}, {"cut_qp_off", s.cut_qp_off.data(), s.cut_qp_off.size(), 1},
      {"qp_wgt", s.qp_wgt.data(), s.qp_wgt.size(), 2}, {"qp_mat", s.qp_mat.data(), s.qp_mat.size(), 1},
      {"qp_grad_off", s.qp_grad_off.data(), s.qp_grad_off.size(), 1}, {"qp_grad", s.qp_grad.data(), s.qp_grad.size(), 2},
      {"cut_coh_off", s.cut_coh_off.data(), s.cut_coh_off.size(), 1}, {"coh_nh", s.coh_nh.data(), s.coh_nh.size(), 1},
      {"coh_local_off", s.coh_local_off.data(), s.coh_local_off.size(), 1}, {"coh_local", s.coh_local.data(), s.coh_local.size(), 1},
      {"coh_qp_off", s.coh_qp_off.data(), s.coh_qp_off.size(), 1}, {"cqp_N", s.cqp_N.data(), s.cqp_N.size(), 2},
      {"cqp_R", s.cqp_R.data(), s.cqp_R.size(), 2}, {"cqp_wgt", s.cqp_wgt.data(), s.cqp_wgt.size(), 2},
      {"cqp_isv", s.cqp_isv.data(), s.cqp_isv.size(), 1}, {"conn", s.conn.data(), s.conn.size(), 1},
      {"elem_mat", s.elem_mat.data(), s.elem_mat.size(), 1}, {"cut_of", s.cut_of.data(), s.cut_of.size(), 1},
      {"node_detect", s.node_detect.data(), s.node_detect.size(), 1}, {"enr_edge", s.enr_edge.data(), s.enr_edge.size(), 1},
      {"enr_incl", s.enr_incl.data(), s.enr_incl.size(), 1}, {"sub_type", s.sub_type.data(), s.sub_type.size(), 1},
      {"cut_sub_off", s.cut_sub_off.data(), s.cut_sub_off.size(), 1}, {"sub_mat", s.sub_mat.data(), s.sub_mat.size(), 1},
      {"fast_dn", c->fast_dn.data(), c->fast_dn.size(), 1}, {"slow_dn", c->slow_dn.data(), c->slow_dn.size(), 1},
      {"dn_node", s.dn_node.data(), s.dn_node.size(), 1}, {"dn_nbr", s.dn_nbr.data(), s.dn_nbr.size(), 1},
      {"dn_nbr_off", s.dn_nbr_off.data(), s.dn_nbr_off.size(), 1}, {"dn_adj", s.dn_adj.data(), s.dn_adj.size(), 1},
      {"dn_adj_off", s.dn_adj_off.data(), s.dn_adj_off.size(), 1},
  };
  for (auto& t : tab)
    if (std::strcmp(t.k, name) == 0) { *n = (int64_t)t.n; *ptr = t.p; return t.kind; }
  *n = 0; *ptr = nullptr;
  return 0;
}

int pg_set_timing(pg_ctx* c, int on) {
  if (!c) return PG_ERR_INPUT;
  c->timing = on != 0;
  return 0;
}

int pg_kernel_times(pg_ctx* c, float* ms) {
  if (!c || !ms || !c->ev[0]) return set_err(c, PG_ERR_STATE, "nothing was launched");
  if (!c->timed_last) return set_err(c, PG_ERR_STATE, "the last assembly ran with timing off (pg_set_timing)");
  if (cudaEventSynchronize(c->ev[5]) != cudaSuccess) return set_err(c, PG_ERR_DEVICE, "event wait failed");
  // [0] cohesive elements and element records, [1] stencil rows (2D: from the start, on their
  // own stream, concurrent with [0] and [2]; 3D: after [0]), [2] general rows (after [0] in 2D,
  // after [1] in 3D), [3] whole assembly
  const bool seq = c->s.dim == 3;
  cudaEventElapsedTime(&ms[0], c->ev[0], c->ev[3]);
  cudaEventElapsedTime(&ms[1], seq ? c->ev[3] : c->ev[0], c->ev[1]);
  cudaEventElapsedTime(&ms[2], seq ? c->ev[1] : c->ev[3], c->ev[4]);
  cudaEventElapsedTime(&ms[3], c->ev[0], c->ev[5]);
  return 0;
}

void pg_destroy(pg_ctx* c) {
  if (!c) return;
  // work of this context still in flight finishes before its memory goes back to the pool
  cudaStreamSynchronize(c->stream);
  if (c->side) cudaStreamSynchronize(c->side);
  if (c->side2) cudaStreamSynchronize(c->side2);
  if (c->pcg.stream) cudaStreamSynchronize(c->pcg.stream);
  if (c->pcg.stream) cudaStreamDestroy(c->pcg.stream);
  if (c->pcg.ev) cudaEventDestroy(c->pcg.ev);
  if (c->pcg.hflag) cudaFreeHost(c->pcg.hflag);
  for (int i = 0; i < 6; ++i) if (c->ev[i]) cudaEventDestroy(c->ev[i]);
  if (c->side) cudaStreamDestroy(c->side);
  if (c->side2) cudaStreamDestroy(c->side2);
  for (void* p : c->allocs) cudaFreeAsync(p, c->up);
  if (c->up) cudaStreamDestroy(c->up);   // released once the frees have run
  delete c->t3c;
  delete c;
}

const char* pg_last_error(const pg_ctx* c) { return c ? c->err.c_str() : "null context"; }

int pg_device_bytes(const pg_ctx* c, int64_t* now, int64_t* peak) {
  if (!c) return PG_ERR_INPUT;
  if (now) *now = (int64_t)c->dev_bytes;
  if (peak) *peak = (int64_t)c->dev_bytes_peak;
  return 0;
}

int pg_get_sizes(const pg_ctx* c, pg_sizes* o) {
  if (!c || !o) return PG_ERR_INPUT;
  const pg::Setup& s = c->s;
  o->dim = s.dim; o->n_nodes = s.n_std + s.n_enr; o->n_std_nodes = s.n_std; o->n_enrich_nodes = s.n_enr;
  o->n_elem = s.ne; o->n_cut_elem = s.ncut; o->n_coh_elem = (int)s.coh_nh.size(); o->n_coh_qp = c->n_coh_qp;
  o->n_free = s.n_free; o->n_const = s.n_const; o->n_isv = s.n_isv;
  for (int b = 0; b < 4; ++b) o->nnz[b] = (int64_t)s.ci[b].size();
  o->cut_scratch_doubles = c->cut_scratch;
  return 0;
}

int pg_get_pattern(const pg_ctx* c, int b, int32_t* rowptr, int32_t* cols) {
  if (!c || b < 0 || b > 3) return PG_ERR_INPUT;
  if (rowptr) std::memcpy(rowptr, c->s.rp[b].data(), c->s.rp[b].size() * sizeof(int32_t));
  if (cols && !c->s.ci[b].empty()) std::memcpy(cols, c->s.ci[b].data(), c->s.ci[b].size() * sizeof(int32_t));
  return 0;
}

int pg_get_nodes(const pg_ctx* c, double* coords, int32_t* node_dofs, double* dirichlet) {
  if (!c) return PG_ERR_INPUT;
  if (coords) std::memcpy(coords, c->s.X.data(), c->s.X.size() * sizeof(double));
  if (node_dofs) std::memcpy(node_dofs, c->s.node_dof.data(), c->s.node_dof.size() * sizeof(int32_t));
  if (dirichlet && !c->s.dirichlet.empty()) std::memcpy(dirichlet, c->s.dirichlet.data(), c->s.dirichlet.size() * sizeof(double));
  return 0;
}

int pg_set_stream(pg_ctx* c, void* stream) {
  if (!c) return PG_ERR_INPUT;
  c->stream = (cudaStream_t)stream;
  return 0;
}

int pg_assemble_device(pg_ctx* c, const double* d_U, double t_frac, int flags) {
  if (!c || !d_U) return PG_ERR_INPUT;
  if (!pg_resident(c)) return set_err(c, PG_ERR_STATE, "the context has no device residency (pg_upload it first)");
  if (reinterpret_cast<uintptr_t>(d_U) % 16) return set_err(c, PG_ERR_INPUT, "the displacement array must be 16-byte aligned");
  if (!(flags & (PG_FUNC | PG_JAC))) return 0;
  double* keep = c->d_U;
  c->d_U = const_cast<double*>(d_U);
  int rc = launch(c, t_frac, flags);
  c->d_U = keep;
  c->assembled = (rc == 0);
  return rc;
}

int pg_residual_strains(pg_ctx* c, const double* d_U, double t_frac, int n_cases, const double* eps, double* d_Rf,
                        double* d_Rp) {
  if (!c || !d_U || !eps || !d_Rf || n_cases < 1 || n_cases > 6) return PG_ERR_INPUT;
  if (!pg_resident(c)) return set_err(c, PG_ERR_STATE, "the context has no device residency (pg_upload it first)");
  if (reinterpret_cast<uintptr_t>(d_U) % 16) return set_err(c, PG_ERR_INPUT, "the displacement array must be 16-byte aligned");
  if (!c->s.desc.subscale) return set_err(c, PG_ERR_INPUT, "macroscale strain cases need a subscale (periodic) problem");
  if (c->s.etype == pg::QUAD4) return set_err(c, PG_ERR_UNSUPPORTED, "the multi-strain pass takes tri3 / tet4 meshes (quad4: one residual-only assembly per strain)");
  if (c->s.n_const > 0 && !d_Rp) return set_err(c, PG_ERR_INPUT, "d_Rp is required when the problem has constrained DOFs");
  pgd::DevProblem P = c->P;
  P.U = d_U;
  P.flags = PG_FUNC;
  for (int v = 0; v < 6; ++v) P.eps_macro[v] = 0.0;
  P.n_cases = n_cases;
  for (int k = 0; k < n_cases; ++k)
    for (int v = 0; v < 6; ++v) P.eps_cases[k][v] = eps[k * 6 + v] * t_frac;
  P.Pf_cases = d_Rf;
  P.Pp_cases = d_Rp;
  const int dim = c->s.dim;
  if (dim == 2) pgl::residual_cases<2>(c, P);
  else pgl::residual_cases<3>(c, P);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_err(c, PG_ERR_DEVICE, std::string("launch failed: ") + cudaGetErrorString(e));
  return 0;
}

int pg_assemble(pg_ctx* c, const double* U, double t_frac, int flags, double* Kff, double* Kfp, double* Kpf, double* Kpp,
                double* Pf, double* Pp) {
  if (!c || !U) return PG_ERR_INPUT;
  if (!pg_resident(c)) return set_err(c, PG_ERR_STATE, "the context has no device residency (pg_upload it first)");
  if (!(flags & (PG_FUNC | PG_JAC))) return 0;
  const pg::Setup& s = c->s;
  const size_t nU = (size_t)(s.n_std + s.n_enr) * s.dim;
  if (cudaMemcpyAsync(c->d_U, U, nU * sizeof(double), cudaMemcpyHostToDevice, c->stream) != cudaSuccess)
    return set_err(c, PG_ERR_DEVICE, "copy of U failed");
  cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream);
  PG_TRY(launch(c, t_frac, flags));
  double* outs[4] = {Kff, Kfp, Kpf, Kpp};
  if (flags & PG_JAC) {
    // PG_KEEP_STATIC with the same host arrays and precision as the last full copy: only the
    // values that can have changed since (a suffix of each block) go back
    const bool fp32 = (flags & PG_FP32) != 0;
    bool keep = (flags & PG_KEEP_STATIC) && c->kept_valid && c->kept_fp32 == fp32;
    for (int b = 0; b < 4; ++b) keep = keep && outs[b] == c->kept[b];
    for (int b = 0; b < 4; ++b) {
      if (!outs[b] || s.ci[b].empty()) continue;
      const long long from = keep ? c->changing_from[b] : 0, nnz = (long long)s.ci[b].size();
      if (from < nnz)
        cudaMemcpyAsync(outs[b] + from, c->P.val[b] + from, (size_t)(nnz - from) * sizeof(double), cudaMemcpyDeviceToHost,
                        c->stream);
    }
    if (flags & PG_KEEP_STATIC) {
      for (int b = 0; b < 4; ++b) c->kept[b] = outs[b];
      c->kept_fp32 = fp32;
      c->kept_valid = true;
    } else {
      c->kept_valid = false;
    }
  }
  if (flags & PG_FUNC) {
    if (Pf && s.n_free) cudaMemcpyAsync(Pf, c->P.Pf, (size_t)s.n_free * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if (Pp && s.n_const) cudaMemcpyAsync(Pp, c->P.Pp, (size_t)s.n_const * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  }
  int herr = 0;
  cudaMemcpyAsync(&herr, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return set_err(c, PG_ERR_DEVICE, std::string("assembly failed: ") + cudaGetErrorString(e));
  c->assembled = true;
  if (herr & pgd::ERR_NONFINITE) return set_err(c, PG_ERR_NONFINITE, "non-finite value in a cut-element matrix or vector");
  if (herr) return set_err(c, PG_ERR_DEVICE, "scatter map inconsistency detected on the device");
  return 0;
}

int pg_changing_values(const pg_ctx* c, int64_t* first) {
  if (!c || !first) return PG_ERR_INPUT;
  for (int b = 0; b < 4; ++b) first[b] = (int64_t)c->changing_from[b];
  return 0;
}

int pg_device_outputs(pg_ctx* c, double** K, double** Pf, double** Pp) {
  if (!c) return PG_ERR_INPUT;
  if (K) for (int b = 0; b < 4; ++b) K[b] = c->P.val[b];
  if (Pf) *Pf = c->P.Pf;
  if (Pp) *Pp = c->P.Pp;
  return 0;
}

int pg_set_isv(pg_ctx* c, const double* v) {
  if (!c || (!v && c->s.n_isv)) return PG_ERR_INPUT;
  if (!pg_resident(c)) return set_err(c, PG_ERR_STATE, "the context has no device residency (pg_upload it first)");
  if (c->s.n_isv == 0) return 0;
  cudaMemcpyAsync(c->d_isv_committed, v, (size_t)c->s.n_isv * sizeof(double), cudaMemcpyHostToDevice, c->stream);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return set_err(c, PG_ERR_DEVICE, "copy of internal variables failed");
  return 0;
}

int pg_get_isv(const pg_ctx* c, int trial, double* out) {
  if (!c || (!out && c->s.n_isv)) return PG_ERR_INPUT;
  if (!pg_resident(c)) return PG_ERR_STATE;
  if (c->s.n_isv == 0) return 0;
  cudaStreamSynchronize(c->stream);
  cudaMemcpyAsync(out, trial ? c->d_isv_trial : c->d_isv_committed, (size_t)c->s.n_isv * sizeof(double), cudaMemcpyDeviceToHost,
                  c->stream);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return PG_ERR_DEVICE;
  return 0;
}

int pg_commit_isv(pg_ctx* c) {
  if (!c) return PG_ERR_INPUT;
  if (!pg_resident(c)) return set_err(c, PG_ERR_STATE, "the context has no device residency (pg_upload it first)");
  if (c->s.n_isv == 0) return 0;
  cudaMemcpyAsync(c->d_isv_committed, c->d_isv_trial, (size_t)c->s.n_isv * sizeof(double), cudaMemcpyDeviceToDevice, c->stream);
  return cudaStreamSynchronize(c->stream) == cudaSuccess ? 0 : PG_ERR_DEVICE;
}

int pg_get_damage_zones(const pg_ctx* c, uint8_t* z) {
  if (!c || (!z && c->n_coh_qp)) return PG_ERR_INPUT;
  if (!pg_resident(c)) return PG_ERR_STATE;
  if (!c->n_coh_qp) return 0;
  cudaStreamSynchronize(c->stream);
  cudaMemcpyAsync(z, c->d_zone, (size_t)c->n_coh_qp, cudaMemcpyDeviceToHost, c->stream);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return PG_ERR_DEVICE;
  return 0;
}

int pg_set_macro_strain(pg_ctx* c, const double* eps) {
  if (!c || !eps) return PG_ERR_INPUT;
  if (!c->s.desc.subscale) return set_err(c, PG_ERR_STATE, "the macroscale strain applies to subscale (periodic) problems only");
  for (int v = 0; v < 6; ++v) c->s.desc.eps_macro[v] = (v < (c->s.dim == 2 ? 3 : 6)) ? eps[v] : 0.0;
  return 0;
}

int pg_residual_norm(pg_ctx* c, double* out) {
  if (!c || !out) return PG_ERR_INPUT;
  if (!pg_resident(c)) return set_err(c, PG_ERR_STATE, "the context has no device residency (pg_upload it first)");
  const int nb = 256;
  k_sumsq_partial<<<nb, 256, 0, c->stream>>>(c->P.Pf, c->s.n_free, c->d_red);
  k_sum_final<<<1, 32, 0, c->stream>>>(c->d_red, nb, c->d_red + nb);
  double v = 0.0;
  cudaMemcpyAsync(&v, c->d_red + nb, sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return set_err(c, PG_ERR_DEVICE, "residual norm failed");
  *out = sqrt(v);
  return 0;
}

}  // extern "C"
