// C ABI of the engine (include/multifil_b200.h): contexts, lattice upload,
// batched / plain execution, host-side jax.random, and the serving loop.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/multifil_b200.h"
#include "mf_kernel.cuh"
#include "mf_launch.cuh"
#include "mf_state.cuh"

using namespace mf;

namespace {

// CTA configuration of a lattice in one precision mode.
struct Cfg {
  int threads = 0;          // CTA size
  bool vec_global = false;  // CG vectors and head terms in the workspace
  bool regs = false;        // register-resident CG layout (x and u only in shared memory)
  size_t smem_local = 0;    // dynamic shared memory at that size
  bool tuned = false;       // set through mf_tune_threads[_mode]
  // launch grouping key and kernel layout flags
  int group_key() const { return threads * 4 + (vec_global ? 1 : 0) + (regs ? 2 : 0); }
  int layout_flags() const { return (vec_global ? FLAG_VEC_GLOBAL : 0) | (regs ? FLAG_REGS : 0); }
};

struct TopoHost {
  TopoDev dev{};          // host copy with device pointers
  TopoDev* d_struct = nullptr;
  std::vector<void*> allocs;
  Cfg cfg[2];             // [0] float32 mode, [1] precise (mixed) mode
};

struct Request;

struct Server;

}  // namespace

struct mf_ctx {
  int device = 0;
  std::string err;
  std::vector<std::unique_ptr<TopoHost>> topos;
  char* ws = nullptr;
  size_t ws_bytes = 0;
  CondDesc* d_cond = nullptr;
  size_t cond_cap = 0;
  int smem_optin = 0;
  int num_sms = 0;
  Server* server = nullptr;
  cudaStream_t cap_stream = nullptr;  // private stream for CUDA-graph capture
  cudaEvent_t cap_event = nullptr;
  // The executable graph of the last chunked batch and the launch list it was
  // captured from: a later batch with the same launches (same shapes, buffers
  // and flags; the descriptor table's contents may differ) replays it.
  cudaGraphExec_t graph_exec = nullptr;
  std::vector<char> graph_sig;
};

static int fail(mf_ctx* c, int code, const char* fmt, ...) {
  if (c) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    c->err = buf;
  }
  return code;
}

// Whether the kernels can store through p: device or managed memory, or
// page-locked host memory mapped into the device address space at the same
// address (cudaHostAlloc under unified addressing; the kernel then writes
// over the bus and no copy is needed).  Pageable host memory is rejected.
static int check_kernel_ptr(mf_ctx* ctx, const void* p, const char* name) {
  cudaPointerAttributes a{};
  const cudaError_t e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    return fail(ctx, MF_ERR_INVALID, "%s: not a CUDA-accessible pointer (%s)", name, cudaGetErrorString(e));
  }
  if (a.type == cudaMemoryTypeUnregistered)
    return fail(ctx, MF_ERR_INVALID, "%s: pageable host memory (the kernels need device or page-locked memory)",
                name);
  if (a.type == cudaMemoryTypeHost && a.devicePointer != p)
    return fail(ctx, MF_ERR_INVALID, "%s: page-locked memory not mapped at the same device address", name);
  return MF_OK;
}

#define CK(call)                                                                        \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess)                                                              \
      return fail(ctx, e_ == cudaErrorMemoryAllocation ? MF_ERR_NOMEM : MF_ERR_CUDA,     \
                  "%s failed: %s", #call, cudaGetErrorString(e_));                      \
  } while (0)

// ---------------------------------------------------------------------------
// kernel dispatch by CTA size and precision (instances in mf_kernels.cu)
// ---------------------------------------------------------------------------
static cudaError_t prepare(int nt, bool precise, bool dyn, size_t smem) {
#define MF_PREPARE_CASE(NT, P, D) \
  if (nt == NT && precise == (P != 0) && dyn == (D != 0)) return prepare_##NT##_##P##_##D(smem);
  MF_FOR_EACH_INSTANCE(MF_PREPARE_CASE)
#undef MF_PREPARE_CASE
  return cudaErrorInvalidValue;
}

static cudaError_t launch(int nt, const StepArgs& a, int grid, int base, size_t smem, cudaStream_t st) {
  const bool precise = (a.flags & FLAG_PRECISE) != 0, dyn = (a.flags & FLAG_DYN) != 0;
  cudaError_t e = prepare(nt, precise, dyn, smem);
  if (e != cudaSuccess) return e;
  cudaGetLastError();  // clear a stale non-sticky error of an earlier, already reported call
#define MF_LAUNCH_CASE(NT, P, D) \
  if (nt == NT && precise == (P != 0) && dyn == (D != 0)) return launch_##NT##_##P##_##D(a, grid, base, smem, st);
  MF_FOR_EACH_INSTANCE(MF_LAUNCH_CASE)
#undef MF_LAUNCH_CASE
  return cudaErrorInvalidValue;
}

// Default CTA size.  Up to 1200 nodes: 384 threads (one warp per filament of
// a 2x2 lattice) in float32 mode, and in precise mode whenever the lattice
// has at most 12 filaments (the register-resident CG then holds one filament
// per warp), else 256 (two per warp).  512 up to 4000 nodes, else 1024.  The
// autotuner measures and overrides.
static int default_threads(const TopoDev& t, bool precise) {
  if (max_filament(t) > 128) return t.n_dof <= 4000 ? 512 : 1024;
  if (t.n_dof <= 1200) return (!precise || t.n_thick + t.n_thin <= 12) ? 384 : 256;
  if (t.n_dof <= 4000) return 512;
  return 1024;
}

// Configuration of a lattice at nt threads: the register layout where the
// register-resident CG covers the lattice (precise mode, allow_regs: batches
// with n_cg > 0), else every CG vector in shared memory, else in the
// workspace.  false when even that does not fit.
static bool make_cfg(const TopoDev& t, int nt, bool precise, bool allow_regs, bool dyn, int smem_optin, Cfg& c,
                     PopShape ps = PopShape()) {
  c.threads = nt;
  if (max_filament(t) > 128 && nt < kWideThreads) return false;  // no code for long filaments below 512
  if (precise && allow_regs && regcg_fits(t, nt)) {
    const size_t sm = smem_bytes(t, nt, LAYOUT_REGS, true, dyn, ps);
    if (sm + kStaticSmem <= (size_t)smem_optin) {
      c.regs = true;
      c.vec_global = false;
      c.smem_local = sm;
      return true;
    }
  }
  c.regs = false;
  c.vec_global = smem_bytes(t, nt, LAYOUT_SMEM, precise, dyn, ps) + kStaticSmem > (size_t)smem_optin;
  c.smem_local = smem_bytes(t, nt, c.vec_global ? LAYOUT_GLOBAL : LAYOUT_SMEM, precise, dyn, ps);
  return c.smem_local + kStaticSmem <= (size_t)smem_optin;
}

// The configuration a batch uses.  With the lattice spacing solved as an
// unknown both transition tables (827 matrix exponentials) are rebuilt every
// step: an untuned default below 512 threads is raised to 512 (measured
// fastest for every lattice of 1x1 to 4x4 in that mode).  false when the
// batch's exact carve (its populations included) fits no layout.
static bool batch_cfg(const TopoHost& t, int pm, bool dyn, int n_cg, PopShape ps, int smem_optin, Cfg& out) {
  Cfg c = t.cfg[pm];  // sized for a dynamic spacing (the larger carve)
  if (dyn && !c.tuned && c.threads < 512) {
    Cfg c5 = c;
    if (make_cfg(t.dev, 512, pm != 0, true, true, smem_optin, c5, ps)) c = c5;
  }
  // the exact carve of this batch: no register layout without CG steps, no
  // spacing derivatives with a fixed spacing, the populations' tables
  Cfg e = c;
  if (!make_cfg(t.dev, c.threads, pm != 0, n_cg > 0, dyn, smem_optin, e, ps)) return false;
  e.tuned = c.tuned;
  out = e;
  return true;
}

extern "C" {

int mf_abi_version(void) { return MF_ABI_VERSION; }

int mf_create(int device, mf_ctx** out) {
  if (!out) return MF_ERR_INVALID;
  mf_ctx* ctx = new mf_ctx();
  ctx->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) {
    *out = nullptr;
    delete ctx;
    return MF_ERR_CUDA;
  }
  cudaDeviceGetAttribute(&ctx->smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
  cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
  *out = ctx;
  return MF_OK;
}

int mf_server_stop(mf_ctx* ctx);

int mf_destroy(mf_ctx* ctx) {
  if (!ctx) return MF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  if (ctx->server) mf_server_stop(ctx);
  for (auto& t : ctx->topos) {
    for (void* p : t->allocs) cudaFree(p);
    if (t->d_struct) cudaFree(t->d_struct);
  }
  if (ctx->ws) cudaFree(ctx->ws);
  if (ctx->d_cond) cudaFree(ctx->d_cond);
  if (ctx->graph_exec) cudaGraphExecDestroy(ctx->graph_exec);
  if (ctx->cap_stream) cudaStreamDestroy(ctx->cap_stream);
  if (ctx->cap_event) cudaEventDestroy(ctx->cap_event);
  delete ctx;
  return MF_OK;
}

const char* mf_last_error(mf_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int mf_upload_topology(mf_ctx* ctx, const mf_topo_desc* d, int32_t* topo_id) {
  if (!ctx || !d || !topo_id) return fail(ctx, MF_ERR_INVALID, "null argument");
  CK(cudaSetDevice(ctx->device));
  const int nth = d->n_thick, ncr = d->n_crowns, nthin = d->n_thin, ns = d->n_sites;
  const int nxb = d->n_xb_per_crown, width = d->max_sites_per_face, nb = d->n_xb_bins;
  if (nth < 1 || ncr < 2 || nthin < 1 || ns < 2 || nxb < 1 || width < 1 || nb < 1)
    return fail(ctx, MF_ERR_INVALID, "bad lattice sizes");
  if (ncr > kMaxFilament || ns > kMaxFilament)
    return fail(ctx, MF_ERR_INVALID, "filaments longer than %d nodes", kMaxFilament);
  const long X = (long)nth * ncr * nxb, S = (long)nthin * ns;
  if (X > 32767 || S > 32767) return fail(ctx, MF_ERR_INVALID, "lattice too large for int16 indices");
  auto t = std::make_unique<TopoHost>();
  TopoDev& td = t->dev;
  td.n_thick = nth; td.n_crowns = ncr; td.n_thin = nthin; td.n_sites = ns;
  td.nxb = nxb; td.width = width; td.n_bins = nb;
  td.total_xbs = (int)X; td.n_sites_total = (int)S; td.n_thick_nodes = nth * ncr;
  td.n_dof = nth * ncr + (int)S;
  td.plan_thick = make_scan_plan(ncr);
  td.plan_thin = make_scan_plan(ns);
  std::vector<int16_t> xb_face(X), face_sites((size_t)nthin * 3 * width), tm_prev(S), tm_next(S);
  std::vector<uint8_t> valid(X), face_n(nthin * 3);
  for (long i = 0; i < X; ++i) {
    const int th = d->xb_to_thin_id[i], fc = d->xb_to_thin_face[i];
    if (th < 0 || th >= nthin || fc < 0 || fc > 2) return fail(ctx, MF_ERR_INVALID, "bad xb target");
    xb_face[i] = (int16_t)(th * 3 + fc);
    valid[i] = d->xb_valid[i] ? 1 : 0;
  }
  for (int f = 0; f < nthin * 3; ++f) {
    const int n = d->n_sites_per_face[f];
    if (n < 0 || n > width) return fail(ctx, MF_ERR_INVALID, "bad face site count");
    face_n[f] = (uint8_t)n;
    const int first = n > 0 ? d->face_to_sites[(size_t)f * width] : 0;
    for (int k = 0; k < width; ++k) {
      int v = k < n ? d->face_to_sites[(size_t)f * width + k] : first;
      if (v < 0 || v >= ns) return fail(ctx, MF_ERR_INVALID, "bad face site index");
      face_sites[(size_t)f * width + k] = (int16_t)v;
    }
  }
  for (long g = 0; g < S; ++g) {
    const int p = d->tm_prev_neighbor[g], q = d->tm_next_neighbor[g];
    if (p < 0 || p >= ns || q < 0 || q >= ns) return fail(ctx, MF_ERR_INVALID, "bad chain neighbour");
    tm_prev[g] = (int16_t)p;
    tm_next[g] = (int16_t)q;
  }
  std::vector<float> thick_c((size_t)nth * ncr), thin_c(S);
  float cmin = INFINITY, cmax = -INFINITY;
  for (int a = 0; a < nth; ++a)
    for (int c = 0; c < ncr; ++c) {
      const size_t i = (size_t)a * ncr + c;
      const double prev = c > 0 ? (double)d->crown_offsets[i - 1] : 0.0;
      thick_c[i] = (float)(((double)d->crown_offsets[i] - prev) - (double)d->crown_rests[i]);
      cmin = std::min(cmin, d->crown_offsets[i]);
      cmax = std::max(cmax, d->crown_offsets[i]);
    }
  for (int a = 0; a < nthin; ++a)
    for (int j = 0; j < ns; ++j) {
      const size_t g = (size_t)a * ns + j;
      const double nxt = j + 1 < ns ? (double)d->binding_offsets[g + 1] : 0.0;
      thin_c[g] = (float)(((double)d->binding_offsets[g] - nxt) - (double)d->binding_rests[g]);
    }
  td.crown_min = cmin;
  td.crown_max = cmax;
  auto up = [&](const void* src, size_t bytes, const void** dst) -> int {
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, bytes < 16 ? 16 : bytes);
    if (e != cudaSuccess) return fail(ctx, MF_ERR_NOMEM, "cudaMalloc(topology): %s", cudaGetErrorString(e));
    t->allocs.push_back(p);
    e = cudaMemcpy(p, src, bytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return fail(ctx, MF_ERR_CUDA, "cudaMemcpy(topology): %s", cudaGetErrorString(e));
    *dst = p;
    return 0;
  };
  int rc = 0;
  rc |= up(xb_face.data(), X * 2, (const void**)&td.xb_face);
  rc |= up(valid.data(), X, (const void**)&td.xb_valid);
  rc |= up(face_sites.data(), face_sites.size() * 2, (const void**)&td.face_sites);
  rc |= up(face_n.data(), face_n.size(), (const void**)&td.face_n);
  rc |= up(tm_prev.data(), S * 2, (const void**)&td.tm_prev);
  rc |= up(tm_next.data(), S * 2, (const void**)&td.tm_next);
  rc |= up(d->crown_offsets, (size_t)nth * ncr * 4, (const void**)&td.crown_off);
  rc |= up(d->crown_rests, (size_t)nth * ncr * 4, (const void**)&td.crown_rest);
  rc |= up(d->binding_offsets, S * 4, (const void**)&td.bind_off);
  rc |= up(d->binding_rests, S * 4, (const void**)&td.bind_rest);
  rc |= up(d->thin_rest_cumsum, S * 4, (const void**)&td.thin_cum);
  rc |= up(d->xb_bin_edges, (size_t)(nb + 1) * 4, (const void**)&td.edges);
  rc |= up(d->xb_bin_centers, (size_t)nb * 4, (const void**)&td.centers);
  rc |= up(thick_c.data(), thick_c.size() * 4, (const void**)&td.thick_c);
  rc |= up(thin_c.data(), thin_c.size() * 4, (const void**)&td.thin_c);
  if (rc) {
    for (void* p : t->allocs) cudaFree(p);
    return rc < 0 ? rc : MF_ERR_CUDA;
  }
  CK(cudaMalloc(&t->d_struct, sizeof(TopoDev)));
  CK(cudaMemcpy(t->d_struct, &td, sizeof(TopoDev), cudaMemcpyHostToDevice));
  for (int p = 0; p < 2; ++p) {
    Cfg& c = t->cfg[p];
    if (!make_cfg(td, default_threads(td, p != 0), p != 0, true, true, ctx->smem_optin, c))
      return fail(ctx, MF_ERR_INVALID, "lattice needs %zu B shared memory (limit %d)", c.smem_local,
                  ctx->smem_optin);
  }
  ctx->topos.push_back(std::move(t));
  *topo_id = (int32_t)ctx->topos.size() - 1;
  return MF_OK;
}

// Choose the CTA size of a lattice (autotuner hook).
int mf_tune_threads_mode(mf_ctx* ctx, int32_t topo_id, int32_t precise, int32_t threads) {
  if (!ctx || topo_id < 0 || topo_id >= (int)ctx->topos.size())
    return fail(ctx, MF_ERR_NOTFOUND, "unknown topology");
  TopoHost& t = *ctx->topos[topo_id];
  const bool reset = threads == 0;  // back to the default (and the dynamic-spacing floor)
  if (reset) threads = default_threads(t.dev, precise != 0);
  if (threads != 128 && threads != 256 && threads != 384 && threads != 512 && threads != 1024)
    return fail(ctx, MF_ERR_INVALID, "threads must be 0, 128, 256, 384, 512 or 1024");
  Cfg c;
  if (!make_cfg(t.dev, threads, precise != 0, true, true, ctx->smem_optin, c))
    return fail(ctx, MF_ERR_INVALID, "does not fit");
  c.tuned = !reset;
  t.cfg[precise ? 1 : 0] = c;
  return MF_OK;
}

int mf_tune_threads(mf_ctx* ctx, int32_t topo_id, int32_t threads) {
  int rc = mf_tune_threads_mode(ctx, topo_id, 0, threads);
  return rc ? rc : mf_tune_threads_mode(ctx, topo_id, 1, threads);
}

static size_t slot_bytes(const TopoDev& t, PopShape ps = PopShape()) {
  const CoefLayout cl = coef_layout(t);
  return slot_layout(t.n_dof, t.total_xbs, t.n_sites_total, t.n_bins, cl.total, ps.kx(), ps.kt()).total;
}

// Subpopulation inputs of a call (mf_batch / mf_state_batch pop_* fields).
struct PopArgs {
  int n_pops, pop_flags, label_stride;
  const float* pop_params;
  const float* pop_frac;
  const int8_t* xb_label;
  const int8_t* tm_label;
};

// Subpopulation shape of a call, checked against every lattice it runs.
static int check_pops(mf_ctx* ctx, const PopArgs& pa, const std::vector<const TopoDev*>& lattices, PopShape& ps) {
  ps = PopShape();
  if (pa.n_pops <= 1) return MF_OK;
  if (pa.n_pops > MF_MAX_POPS) return fail(ctx, MF_ERR_INVALID, "n_pops %d above %d", pa.n_pops, MF_MAX_POPS);
  if (pa.pop_flags & ~(MF_POP_EXPLICIT | MF_POP_XB | MF_POP_TM))
    return fail(ctx, MF_ERR_INVALID, "unknown pop_flags bits");
  ps.K = pa.n_pops;
  ps.flags = pa.pop_flags;
  if (!ps.active()) return MF_OK;
  if (!pa.pop_params) return fail(ctx, MF_ERR_INVALID, "subpopulations need pop_params");
  if ((ps.blend_xb() || ps.blend_tm()) && !pa.pop_frac)
    return fail(ctx, MF_ERR_INVALID, "mean-field subpopulations need pop_frac");
  if (ps.kx() > 1 && !pa.xb_label) return fail(ctx, MF_ERR_INVALID, "explicit crossbridge populations need xb_label");
  if (ps.kt() > 1 && !pa.tm_label) return fail(ctx, MF_ERR_INVALID, "explicit tropomyosin populations need tm_label");
  for (const TopoDev* td : lattices) {
    if ((ps.kx() > 1 && pa.label_stride < td->total_xbs) || (ps.kt() > 1 && pa.label_stride < td->n_sites_total))
      return fail(ctx, MF_ERR_INVALID, "label_stride %d below a condition's head or site count", pa.label_stride);
    if ((long)ps.kx() * 2 * td->n_bins > 32767) return fail(ctx, MF_ERR_INVALID, "too many population table keys");
  }
  return MF_OK;
}

static int batch_pops(mf_ctx* ctx, const mf_batch* bt, PopShape& ps) {
  std::vector<const TopoDev*> lat;
  if (bt->n_pops > 1)
    for (int i = 0; i < bt->B; ++i) {
      const int id = bt->topo_id[i];
      if (id < 0 || id >= (int)ctx->topos.size()) return fail(ctx, MF_ERR_NOTFOUND, "unknown topology %d", id);
      lat.push_back(&ctx->topos[id]->dev);
    }
  const PopArgs pa{bt->n_pops, bt->pop_flags, bt->label_stride, bt->pop_params, bt->pop_frac, bt->xb_label,
                   bt->tm_label};
  return check_pops(ctx, pa, lat, ps);
}

// Population inputs of condition i in its descriptor.
static void fill_pops(CondDesc& c, const mf_batch* bt, const PopShape& ps, int i) {
  c.pop_params = c.pop_frac = nullptr;
  c.xb_label = c.tm_label = nullptr;
  if (!ps.active()) return;
  c.pop_params = bt->pop_params + (size_t)i * ps.K * MF_N_PARAMS;
  if (bt->pop_frac) c.pop_frac = bt->pop_frac + (size_t)i * ps.K;
  if (ps.kx() > 1) c.xb_label = bt->xb_label + (size_t)i * bt->label_stride;
  if (ps.kt() > 1) c.tm_label = bt->tm_label + (size_t)i * bt->label_stride;
}

int mf_workspace_bytes(mf_ctx* ctx, const mf_batch* bt, uint64_t* bytes) {
  if (!ctx || !bt || !bytes) return fail(ctx, MF_ERR_INVALID, "null argument");
  PopShape ps;
  const int prc = batch_pops(ctx, bt, ps);
  if (prc) return prc;
  uint64_t tot = 0;
  for (int i = 0; i < bt->B; ++i) {
    const int id = bt->topo_id[i];
    if (id < 0 || id >= (int)ctx->topos.size()) return fail(ctx, MF_ERR_NOTFOUND, "unknown topology %d", id);
    tot += slot_bytes(ctx->topos[id]->dev, ps);
  }
  *bytes = tot + sizeof(CondDesc) * (uint64_t)bt->B;
  return MF_OK;
}

static int ensure_ws(mf_ctx* ctx, size_t bytes) {
  if (bytes <= ctx->ws_bytes) return MF_OK;
  if (ctx->ws) cudaFree(ctx->ws);
  ctx->ws = nullptr;
  ctx->ws_bytes = 0;
  size_t want = std::max(bytes, ctx->ws_bytes * 3 / 2);
  cudaError_t e = cudaMalloc(&ctx->ws, want);
  if (e != cudaSuccess) {
    e = cudaMalloc(&ctx->ws, bytes);
    if (e != cudaSuccess) return fail(ctx, MF_ERR_NOMEM, "workspace of %zu B: %s", bytes, cudaGetErrorString(e));
    want = bytes;
  }
  ctx->ws_bytes = want;
  return MF_OK;
}

static int ensure_cond(mf_ctx* ctx, size_t n) {
  if (n <= ctx->cond_cap) return MF_OK;
  if (ctx->d_cond) cudaFree(ctx->d_cond);
  ctx->d_cond = nullptr;
  size_t cap = std::max(n, ctx->cond_cap * 2);
  cudaError_t e = cudaMalloc(&ctx->d_cond, cap * sizeof(CondDesc));
  if (e != cudaSuccess) return fail(ctx, MF_ERR_NOMEM, "condition table: %s", cudaGetErrorString(e));
  ctx->cond_cap = cap;
  return MF_OK;
}

static StepArgs make_args(const mf_batch* bt, const CondDesc* dc, int flags, int max_dof, int max_x,
                          int max_s, PopShape ps) {
  StepArgs a{};
  a.pop = ps;
  a.cond = dc;
  a.T = bt->T_max;
  a.n_newton = bt->n_newton;
  a.n_cg = bt->n_cg;
  a.flags = flags;
  a.resid_warn = bt->residual_warn;
  a.sq64_from = (flags & FLAG_PRECISE) ? 1 : 1 << 20;
  a.u_thin = bt->u_thin;
  a.u_xb = bt->u_xb;
  a.x_trace = bt->x_trace;
  a.st_trace = bt->state_trace;
  a.bd_trace = bt->bound_trace;
  a.max_dof = max_dof;
  a.max_xbs = max_x;
  a.max_sites = max_s;
  return a;
}

int mf_run_batch(mf_ctx* ctx, const mf_batch* bt, void* stream_v) {
  if (!ctx || !bt) return fail(ctx, MF_ERR_INVALID, "null argument");
  if (bt->B < 0 || bt->T_max < 0) return fail(ctx, MF_ERR_INVALID, "negative batch shape");
  if (bt->B == 0) return MF_OK;
  if (!bt->topo_id || !bt->params || !bt->z || !bt->pCa || !bt->ls || !bt->n_steps || !bt->keys ||
      !bt->metrics_out)
    return fail(ctx, MF_ERR_INVALID, "missing required array");
  if (bt->n_newton < 0 || bt->n_cg < 0) return fail(ctx, MF_ERR_INVALID, "negative solver caps");
  if ((bt->flags & MF_FLAG_DYNAMIC_LS) && (!bt->K_lat || !bt->nu))
    return fail(ctx, MF_ERR_INVALID, "dynamic lattice spacing needs K_lat and nu");
  PopShape ps;
  int rc = batch_pops(ctx, bt, ps);
  if (rc) return rc;
  CK(cudaSetDevice(ctx->device));
  if ((rc = check_kernel_ptr(ctx, bt->metrics_out, "metrics_out"))) return rc;
  cudaStream_t st = (cudaStream_t)stream_v;
  const int B = bt->B;
  // group conditions by CTA configuration; one launch per group
  std::vector<int> n_steps(B);
  std::vector<float> h_K(B, 0.f), h_nu(B, 0.f), h_dt(B, 1.0f);
  CK(cudaMemcpy(n_steps.data(), bt->n_steps, sizeof(int) * B, cudaMemcpyDeviceToHost));
  if (bt->K_lat) CK(cudaMemcpy(h_K.data(), bt->K_lat, sizeof(float) * B, cudaMemcpyDeviceToHost));
  if (bt->nu) CK(cudaMemcpy(h_nu.data(), bt->nu, sizeof(float) * B, cudaMemcpyDeviceToHost));
  if (bt->dt) CK(cudaMemcpy(h_dt.data(), bt->dt, sizeof(float) * B, cudaMemcpyDeviceToHost));
  std::vector<CondDesc> hc(B);
  size_t off = 0;
  int max_dof = 0, max_x = 0, max_s = 0;
  for (int i = 0; i < B; ++i) {
    const int id = bt->topo_id[i];
    if (id < 0 || id >= (int)ctx->topos.size()) return fail(ctx, MF_ERR_NOTFOUND, "unknown topology %d", id);
    if (n_steps[i] < 0 || n_steps[i] > bt->T_max) return fail(ctx, MF_ERR_INVALID, "n_steps out of range");
    const TopoDev& td = ctx->topos[id]->dev;
    max_dof = std::max(max_dof, td.n_dof);
    max_x = std::max(max_x, td.total_xbs);
    max_s = std::max(max_s, td.n_sites_total);
    off += slot_bytes(td, ps);
  }
  // CTA configuration of every condition
  const int pm = (bt->flags & MF_FLAG_PRECISE) ? 1 : 0;
  const bool dynb = (bt->flags & MF_FLAG_DYNAMIC_LS) != 0;
  std::vector<Cfg> cfgs(B);
  for (int i = 0; i < B; ++i)
    if (!batch_cfg(*ctx->topos[bt->topo_id[i]], pm, dynb, bt->n_cg, ps, ctx->smem_optin, cfgs[i]))
      return fail(ctx, MF_ERR_INVALID, "condition %d: its lattice and populations exceed shared memory", i);
  rc = ensure_ws(ctx, off);
  if (rc) return rc;
  // order: group by (threads, vec_global), longest work first inside a group
  std::vector<int> order(B);
  for (int i = 0; i < B; ++i) order[i] = i;
  auto key_of = [&](int i) {
    const TopoHost& t = *ctx->topos[bt->topo_id[i]];
    return std::make_pair(cfgs[i].group_key(), -(long)n_steps[i] * t.dev.n_dof);
  };
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return key_of(a) < key_of(b); });
  off = 0;
  for (int k = 0; k < B; ++k) {
    const int i = order[k];
    const TopoHost& t = *ctx->topos[bt->topo_id[i]];
    hc[k].topo = t.d_struct;
    hc[k].ws = ctx->ws + off;
    hc[k].n_steps = n_steps[i];
    hc[k].index = i;
    hc[k].T = bt->T_max;
    hc[k].t0 = 0;
    hc[k].t1 = n_steps[i];
    hc[k].params = bt->params + (size_t)i * MF_N_PARAMS;
    const size_t dstride = (bt->flags & MF_FLAG_CONST_DRIVERS) ? 1 : (size_t)bt->T_max;
    hc[k].drv_const = (bt->flags & MF_FLAG_CONST_DRIVERS) ? 1 : 0;
    hc[k].z = bt->z + (size_t)i * dstride;
    hc[k].pCa = bt->pCa + (size_t)i * dstride;
    hc[k].ls = bt->ls + (size_t)i * dstride;
    hc[k].key = bt->keys + 2 * (size_t)i;
    hc[k].metrics = bt->metrics_out + (size_t)i * MF_N_METRICS * bt->T_max;
    hc[k].status = bt->status_out ? bt->status_out + i : nullptr;
    hc[k].key_out = bt->keys_out ? bt->keys_out + 2 * (size_t)i : nullptr;
    hc[k].K_lat = h_K[i];
    hc[k].nu = h_nu[i];
    hc[k].dt = h_dt[i];
    fill_pops(hc[k], bt, ps, i);
    off += slot_bytes(t.dev, ps);
  }
  int base_flags = 0;
  if (bt->flags & MF_FLAG_DYNAMIC_LS) base_flags |= FLAG_DYN;
  if (bt->flags & MF_FLAG_PRECISE) base_flags |= FLAG_PRECISE;
  if (bt->flags & MF_FLAG_ORIGINAL_PRNG) base_flags |= FLAG_ORIG_PRNG;
  int T = 0;
  for (int i = 0; i < B; ++i) T = std::max(T, n_steps[i]);
  // groups
  struct Group { int begin, end, threads, key, lflags; size_t smem; };
  std::vector<Group> groups;
  for (int k = 0; k < B;) {
    const Cfg& c0 = cfgs[order[k]];
    Group g{k, k, c0.threads, c0.group_key(), c0.layout_flags(), 0};
    while (g.end < B) {
      const Cfg& ck = cfgs[order[g.end]];
      if (ck.group_key() != g.key) break;
      g.smem = std::max(g.smem, ck.smem_local);
      ++g.end;
    }
    groups.push_back(g);
    k = g.end;
  }
  const bool plain = (bt->flags & MF_FLAG_PLAIN) != 0;
  if (plain) {
    // One condition per launch, one launch per step: every step reloads the
    // condition from its resident workspace and stores it back.  The step
    // range of each launch is baked into its own descriptor row.
    size_t n_rows = 0;
    for (int k = 0; k < B; ++k) n_rows += (size_t)std::max(hc[k].n_steps, 1);
    rc = ensure_cond(ctx, n_rows + B);
    if (rc) return rc;
    std::vector<CondDesc> rows;
    rows.reserve(n_rows);
    std::vector<std::pair<int, int>> launches;  // (row, group)
    for (size_t gi = 0; gi < groups.size(); ++gi)
      for (int k = groups[gi].begin; k < groups[gi].end; ++k)
        for (int t = 0; t < std::max(hc[k].n_steps, 1); ++t) {
          CondDesc c = hc[k];
          c.t0 = t;
          c.t1 = t + 1;
          launches.emplace_back((int)rows.size(), (int)gi);
          rows.push_back(c);
        }
    CK(cudaMemcpyAsync(ctx->d_cond, rows.data(), sizeof(CondDesc) * rows.size(), cudaMemcpyHostToDevice, st));
    for (auto& lr : launches) {
      const Group& g = groups[lr.second];
      StepArgs a = make_args(bt, ctx->d_cond, base_flags | g.lflags, max_dof, max_x, max_s, ps);
      cudaError_t e = launch(g.threads, a, 1, lr.first, g.smem, st);
      if (e != cudaSuccess) return fail(ctx, MF_ERR_CUDA, "plain launch: %s", cudaGetErrorString(e));
    }
    CK(cudaStreamSynchronize(st));  // the host staging vector dies here
    return MF_OK;
  }
  const int chunk = bt->chunk_steps > 0 ? bt->chunk_steps : std::max(T, 1);
  const int n_chunks = (std::max(T, 1) + chunk - 1) / chunk;
  // one descriptor table per chunk (step ranges differ), uploaded once
  rc = ensure_cond(ctx, (size_t)B * n_chunks);
  if (rc) return rc;
  std::vector<CondDesc> tab((size_t)B * n_chunks);
  for (int c = 0; c < n_chunks; ++c)
    for (int k = 0; k < B; ++k) {
      CondDesc d = hc[k];
      d.t0 = c * chunk;
      d.t1 = std::min(c * chunk + chunk, d.n_steps);
      tab[(size_t)c * B + k] = d;
    }
  CK(cudaMemcpyAsync(ctx->d_cond, tab.data(), sizeof(CondDesc) * tab.size(), cudaMemcpyHostToDevice, st));
  // the launches of the whole batch: every chunk, every CTA-size group
  struct Launch { int threads, grid, base; size_t smem; StepArgs args; };
  std::vector<Launch> launches;
  for (int c = 0; c < n_chunks; ++c)
    for (const Group& g : groups)
      launches.push_back({g.threads, g.end - g.begin, g.begin, g.smem,
                          make_args(bt, ctx->d_cond + (size_t)c * B, base_flags | g.lflags, max_dof, max_x, max_s,
                                    ps)});
  const bool use_graph = !(bt->flags & MF_FLAG_NO_GRAPH) && n_chunks > 1;
  if (!use_graph) {
    for (const Launch& l : launches) {
      cudaError_t e = launch(l.threads, l.args, l.grid, l.base, l.smem, st);
      if (e != cudaSuccess) return fail(ctx, MF_ERR_CUDA, "launch: %s", cudaGetErrorString(e));
    }
    CK(cudaStreamSynchronize(st));  // the host descriptor table dies here
    return MF_OK;
  }
  // Chunked batches replay one CUDA graph of all their launches.  The launch
  // list, field by field, is the graph's signature.
  std::vector<char> sig;
  auto put = [&sig](const void* p, size_t n) {
    const char* c = static_cast<const char*>(p);
    sig.insert(sig.end(), c, c + n);
  };
  for (const Launch& l : launches) {
    const StepArgs& a = l.args;
    put(&l.threads, sizeof l.threads); put(&l.grid, sizeof l.grid); put(&l.base, sizeof l.base);
    put(&l.smem, sizeof l.smem); put(&a.cond, sizeof a.cond); put(&a.T, sizeof a.T);
    put(&a.n_newton, sizeof a.n_newton); put(&a.n_cg, sizeof a.n_cg); put(&a.flags, sizeof a.flags);
    put(&a.resid_warn, sizeof a.resid_warn); put(&a.sq64_from, sizeof a.sq64_from);
    put(&a.u_thin, sizeof a.u_thin); put(&a.u_xb, sizeof a.u_xb); put(&a.x_trace, sizeof a.x_trace);
    put(&a.st_trace, sizeof a.st_trace); put(&a.bd_trace, sizeof a.bd_trace); put(&a.max_dof, sizeof a.max_dof);
    put(&a.max_xbs, sizeof a.max_xbs); put(&a.max_sites, sizeof a.max_sites);
    put(&a.pop.K, sizeof a.pop.K); put(&a.pop.flags, sizeof a.pop.flags);
  }
  if (!ctx->graph_exec || sig != ctx->graph_sig) {
    // capture on a private non-blocking stream (the caller's may be the legacy
    // default stream, which cannot be captured); the graph replays on st
    if (!ctx->cap_stream) {
      CK(cudaStreamCreateWithFlags(&ctx->cap_stream, cudaStreamNonBlocking));
      CK(cudaEventCreateWithFlags(&ctx->cap_event, cudaEventDisableTiming));
    }
    if (ctx->graph_exec) {
      cudaGraphExecDestroy(ctx->graph_exec);
      ctx->graph_exec = nullptr;
      ctx->graph_sig.clear();
    }
    cudaStream_t cs = ctx->cap_stream;
    for (const Group& g : groups)
      CK(prepare(g.threads, (base_flags & FLAG_PRECISE) != 0, (base_flags & FLAG_DYN) != 0, g.smem));
    CK(cudaEventRecord(ctx->cap_event, st));
    CK(cudaStreamWaitEvent(cs, ctx->cap_event, 0));
    CK(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    cudaGraph_t graph = nullptr;
    for (const Launch& l : launches) {
      cudaError_t e = launch(l.threads, l.args, l.grid, l.base, l.smem, cs);
      if (e != cudaSuccess) {
        cudaStreamEndCapture(cs, &graph);
        if (graph) cudaGraphDestroy(graph);
        return fail(ctx, MF_ERR_CUDA, "launch: %s", cudaGetErrorString(e));
      }
    }
    CK(cudaStreamEndCapture(cs, &graph));
    cudaGraphExec_t exec = nullptr;
    cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail(ctx, MF_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
    ctx->graph_exec = exec;
    ctx->graph_sig.swap(sig);
  }
  {
    cudaError_t e = cudaGraphLaunch(ctx->graph_exec, st);
    if (e != cudaSuccess) return fail(ctx, MF_ERR_CUDA, "graph launch: %s", cudaGetErrorString(e));
  }
  CK(cudaStreamSynchronize(st));  // the host descriptor table dies here
  return MF_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Test hook: the transition tables of one (parameter row, pCa, spacing, dt).
// ---------------------------------------------------------------------------
namespace {

// One CTA builds every table with the step kernel's own builder.
__global__ void tables_probe_kernel(const float* params, const float* centers, int nb, float pCa, float d,
                                    float dt, int sq64, float* cum_tm, float* cum_xb, float* pabs) {
  __shared__ float P[kNParams];
  __shared__ TableCtx tc;
  for (int i = threadIdx.x; i < kNParams; i += blockDim.x) P[i] = params[i];
  if (threadIdx.x == 0) {
    tc.P = P;
    tc.centers = centers;
    tc.nb = nb;
    tc.dtm = dt;
    tc.sq64 = sq64;
    tc.cum_tm = cum_tm;
    tc.cum_xb = cum_xb;
    tc.pabs = pabs;
    tc.pop = PopShape();
    tc.Pk = tc.fk = nullptr;
  }
  __syncthreads();
  build_tables_block(tc, pCa, d, true, true, true, nullptr, 0, (int)threadIdx.x, (int)blockDim.x);
}

}  // namespace

extern "C" {

int mf_transition_tables(mf_ctx* ctx, int32_t topo_id, const float* params, float pCa, float d, float dt,
                         int32_t flags, float* cum_tm, float* cum_xb, float* pabs) {
  if (!ctx || !params) return fail(ctx, MF_ERR_INVALID, "null argument");
  if (topo_id < 0 || topo_id >= (int)ctx->topos.size()) return fail(ctx, MF_ERR_NOTFOUND, "unknown topology");
  CK(cudaSetDevice(ctx->device));
  const TopoDev& td = ctx->topos[topo_id]->dev;
  const int nb = td.n_bins;
  const size_t n_tm = 27 * 16, n_xb = (size_t)2 * nb * 36, n_abs = (size_t)2 * nb * 3;
  float* buf = nullptr;
  CK(cudaMalloc(&buf, sizeof(float) * (kNParams + n_tm + n_xb + n_abs)));
  float *dp = buf, *dtm = buf + kNParams, *dxb = dtm + n_tm, *dab = dxb + n_xb;
  const int sq64 = (flags & MF_FLAG_PRECISE) ? 1 : 1 << 20;  // as make_args
  cudaError_t e = cudaMemcpy(dp, params, sizeof(float) * kNParams, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    tables_probe_kernel<<<1, 256>>>(dp, td.centers, nb, pCa, d, dt, sq64, dtm, dxb, dab);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e == cudaSuccess && cum_tm) e = cudaMemcpy(cum_tm, dtm, sizeof(float) * n_tm, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && cum_xb) e = cudaMemcpy(cum_xb, dxb, sizeof(float) * n_xb, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && pabs) e = cudaMemcpy(pabs, dab, sizeof(float) * n_abs, cudaMemcpyDeviceToHost);
  cudaFree(buf);
  if (e != cudaSuccess) return fail(ctx, MF_ERR_CUDA, "mf_transition_tables: %s", cudaGetErrorString(e));
  return MF_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free batch entry point.
//
// mf_run_batch grows a library-owned workspace with cudaMalloc whenever a
// batch needs more room than it has.  Some callers cannot accept that: a host
// framework that hands every byte of HBM to its own allocator and budget, or
// a latency-critical loop for which cudaMalloc's implicit device-wide
// synchronisation is a stall.  mf_run_batch_static serves them by taking all
// of its per-call device memory -- the per-condition resident workspaces and
// the launch descriptor table -- from one fixed array compiled into this
// library (kStaticScratchBytes per device, resident in every process that
// loads the library, for the life of that process).  It never calls
// cudaMalloc, cudaFree or any allocating routine.
// ---------------------------------------------------------------------------
namespace {

constexpr size_t kStaticScratchBytes = size_t(8) << 20;  // 8 MiB per device
constexpr int kMaxDevices = 64;

static __device__ __align__(256) char g_static_scratch[kStaticScratchBytes];

// Device address of g_static_scratch per device, resolved once with that
// device current (the host symbol itself is not a device address).  The
// once-flag makes two host threads' first calls on one device resolve it
// once; the result code is kept so that a failed resolution is reported to
// every later call instead of being retried.
char* g_static_ptr[kMaxDevices] = {nullptr};
cudaError_t g_static_err[kMaxDevices] = {};
std::once_flag g_static_once[kMaxDevices];

}  // namespace

extern "C" {

int mf_run_batch_static(mf_ctx* ctx, const mf_batch* bt, void* stream_v) {
  if (!ctx || !bt) return fail(ctx, MF_ERR_INVALID, "null argument");
  if (bt->B < 0 || bt->T_max < 0) return fail(ctx, MF_ERR_INVALID, "negative batch shape");
  if (bt->B == 0) return MF_OK;
  if (!bt->topo_id || !bt->params || !bt->z || !bt->pCa || !bt->ls || !bt->n_steps || !bt->keys ||
      !bt->metrics_out)
    return fail(ctx, MF_ERR_INVALID, "missing required array");
  if (bt->flags & (MF_FLAG_PLAIN)) return fail(ctx, MF_ERR_INVALID, "mf_run_batch_static: plain path not offered");
  if (bt->chunk_steps > 0) return fail(ctx, MF_ERR_INVALID, "mf_run_batch_static: runs all steps in one launch");
  if ((bt->flags & MF_FLAG_DYNAMIC_LS) && (!bt->K_lat || !bt->nu))
    return fail(ctx, MF_ERR_INVALID, "dynamic lattice spacing needs K_lat and nu");
  if (bt->n_newton < 0 || bt->n_cg < 0) return fail(ctx, MF_ERR_INVALID, "negative solver caps");
  if (ctx->device < 0 || ctx->device >= kMaxDevices) return fail(ctx, MF_ERR_INVALID, "device index out of range");
  PopShape ps;
  {
    const int prc = batch_pops(ctx, bt, ps);
    if (prc) return prc;
  }
  CK(cudaSetDevice(ctx->device));
  {
    const int prc = check_kernel_ptr(ctx, bt->metrics_out, "metrics_out");
    if (prc) return prc;
  }
  // one-time set-up on this device, with the device current
  const int dev = ctx->device;
  std::call_once(g_static_once[dev], [dev]() {
    void* p = nullptr;
    g_static_err[dev] = cudaGetSymbolAddress(&p, g_static_scratch);
    if (g_static_err[dev] == cudaSuccess && !p) g_static_err[dev] = cudaErrorInvalidSymbol;
    if (g_static_err[dev] == cudaSuccess) g_static_ptr[dev] = static_cast<char*>(p);
  });
  if (g_static_err[dev] != cudaSuccess)
    return fail(ctx, MF_ERR_CUDA, "cudaGetSymbolAddress(static scratch): %s", cudaGetErrorString(g_static_err[dev]));
  char* base = g_static_ptr[dev];
  cudaStream_t st = (cudaStream_t)stream_v;
  const int B = bt->B;
  std::vector<int> n_steps(B);
  std::vector<float> h_K(B, 0.f), h_nu(B, 0.f), h_dt(B, 1.0f);
  CK(cudaMemcpy(n_steps.data(), bt->n_steps, sizeof(int) * B, cudaMemcpyDeviceToHost));
  if (bt->K_lat) CK(cudaMemcpy(h_K.data(), bt->K_lat, sizeof(float) * B, cudaMemcpyDeviceToHost));
  if (bt->nu) CK(cudaMemcpy(h_nu.data(), bt->nu, sizeof(float) * B, cudaMemcpyDeviceToHost));
  if (bt->dt) CK(cudaMemcpy(h_dt.data(), bt->dt, sizeof(float) * B, cudaMemcpyDeviceToHost));
  // size check: descriptor table + every condition's workspace must fit
  const size_t desc_bytes = align_up(sizeof(CondDesc) * (size_t)B, 256);
  size_t need = desc_bytes;
  int max_dof = 0, max_x = 0, max_s = 0;
  for (int i = 0; i < B; ++i) {
    const int id = bt->topo_id[i];
    if (id < 0 || id >= (int)ctx->topos.size()) return fail(ctx, MF_ERR_NOTFOUND, "unknown topology %d", id);
    if (n_steps[i] < 0 || n_steps[i] > bt->T_max) return fail(ctx, MF_ERR_INVALID, "n_steps out of range");
    const TopoDev& td = ctx->topos[id]->dev;
    max_dof = std::max(max_dof, td.n_dof);
    max_x = std::max(max_x, td.total_xbs);
    max_s = std::max(max_s, td.n_sites_total);
    need += slot_bytes(td, ps);
  }
  if (need > kStaticScratchBytes)
    return fail(ctx, MF_ERR_NOMEM,
                "mf_run_batch_static: batch needs %zu B of scratch, the static array holds %zu B "
                "(split the batch or use mf_run_batch)", need, kStaticScratchBytes);
  // group by CTA configuration exactly as mf_run_batch does
  const int pm = (bt->flags & MF_FLAG_PRECISE) ? 1 : 0;
  const bool dynb = (bt->flags & MF_FLAG_DYNAMIC_LS) != 0;
  std::vector<Cfg> cfgs(B);
  for (int i = 0; i < B; ++i)
    if (!batch_cfg(*ctx->topos[bt->topo_id[i]], pm, dynb, bt->n_cg, ps, ctx->smem_optin, cfgs[i]))
      return fail(ctx, MF_ERR_INVALID, "condition %d: its lattice and populations exceed shared memory", i);
  std::vector<int> order(B);
  for (int i = 0; i < B; ++i) order[i] = i;
  auto key_of = [&](int i) {
    const TopoHost& t = *ctx->topos[bt->topo_id[i]];
    return std::make_pair(cfgs[i].group_key(), -(long)n_steps[i] * t.dev.n_dof);
  };
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return key_of(a) < key_of(b); });
  CondDesc* d_desc = reinterpret_cast<CondDesc*>(base);
  std::vector<CondDesc> hc(B);
  size_t off = desc_bytes;
  for (int k = 0; k < B; ++k) {
    const int i = order[k];
    const TopoHost& t = *ctx->topos[bt->topo_id[i]];
    CondDesc& c = hc[k];
    c.topo = t.d_struct;
    c.ws = base + off;
    c.n_steps = n_steps[i];
    c.index = i;
    c.T = bt->T_max;
    c.t0 = 0;
    c.t1 = n_steps[i];
    c.params = bt->params + (size_t)i * MF_N_PARAMS;
    const size_t dstride = (bt->flags & MF_FLAG_CONST_DRIVERS) ? 1 : (size_t)bt->T_max;
    c.drv_const = (bt->flags & MF_FLAG_CONST_DRIVERS) ? 1 : 0;
    c.z = bt->z + (size_t)i * dstride;
    c.pCa = bt->pCa + (size_t)i * dstride;
    c.ls = bt->ls + (size_t)i * dstride;
    c.key = bt->keys + 2 * (size_t)i;
    c.metrics = bt->metrics_out + (size_t)i * MF_N_METRICS * bt->T_max;
    c.status = bt->status_out ? bt->status_out + i : nullptr;
    c.key_out = bt->keys_out ? bt->keys_out + 2 * (size_t)i : nullptr;
    c.K_lat = h_K[i];
    c.nu = h_nu[i];
    c.dt = h_dt[i];
    fill_pops(c, bt, ps, i);
    off += slot_bytes(t.dev, ps);
  }
  // The array keeps whatever the previous call left.  The kernel rebuilds
  // every workspace field at step 0, but the region this call uses is zeroed
  // first so no stale byte can ever be read.  Calls whose work overlaps on
  // the GPU (different streams, or no ordering between them) share this one
  // array and race; callers must serialise them.
  CK(cudaMemsetAsync(base, 0, off, st));
  CK(cudaMemcpyAsync(d_desc, hc.data(), sizeof(CondDesc) * B, cudaMemcpyHostToDevice, st));
  int flags = 0;
  if (bt->flags & MF_FLAG_DYNAMIC_LS) flags |= FLAG_DYN;
  if (bt->flags & MF_FLAG_PRECISE) flags |= FLAG_PRECISE;
  if (bt->flags & MF_FLAG_ORIGINAL_PRNG) flags |= FLAG_ORIG_PRNG;
  for (int k = 0; k < B;) {
    const Cfg& c0 = cfgs[order[k]];
    int e = k;
    size_t smem = 0;
    while (e < B) {
      const Cfg& ck = cfgs[order[e]];
      if (ck.group_key() != c0.group_key()) break;
      smem = std::max(smem, ck.smem_local);
      ++e;
    }
    StepArgs a = make_args(bt, d_desc, flags | c0.layout_flags(), max_dof, max_x, max_s, ps);
    cudaError_t err = launch(c0.threads, a, e - k, k, smem, st);
    if (err != cudaSuccess) return fail(ctx, MF_ERR_CUDA, "static launch: %s", cudaGetErrorString(err));
    k = e;
  }
  CK(cudaStreamSynchronize(st));  // the host descriptor staging vector dies here
  return MF_OK;
}

// ---------------------------------------------------------------------------
// One step of caller-owned states (state_kernel, mf_state.cuh).
// ---------------------------------------------------------------------------
static cudaError_t prepare_state(int nt, bool dyn, size_t smem) {
#define MF_PREP_STATE_CASE(NT, D) \
  if (nt == NT && dyn == (D != 0)) return prepare_state_##NT##_##D(smem);
  MF_FOR_EACH_STATE_INSTANCE(MF_PREP_STATE_CASE)
#undef MF_PREP_STATE_CASE
  return cudaErrorInvalidValue;
}

static cudaError_t launch_state(int nt, bool dyn, const StepArgs& a, const StateIO& io, int grid, size_t smem,
                                cudaStream_t st) {
  cudaError_t e = prepare_state(nt, dyn, smem);
  if (e != cudaSuccess) return e;
  cudaGetLastError();
#define MF_LAUNCH_STATE_CASE(NT, D) \
  if (nt == NT && dyn == (D != 0)) return launch_state_##NT##_##D(a, io, grid, smem, st);
  MF_FOR_EACH_STATE_INSTANCE(MF_LAUNCH_STATE_CASE)
#undef MF_LAUNCH_STATE_CASE
  return cudaErrorInvalidValue;
}

int mf_step_states(mf_ctx* ctx, const mf_state_batch* sb, void* stream_v) {
  if (!ctx || !sb) return fail(ctx, MF_ERR_INVALID, "null argument");
  if (sb->B < 0) return fail(ctx, MF_ERR_INVALID, "negative batch size");
  if (sb->B == 0) return MF_OK;
  if (sb->topo_id < 0 || sb->topo_id >= (int)ctx->topos.size()) return fail(ctx, MF_ERR_NOTFOUND, "unknown topology");
  if (sb->phases & ~(MF_PHASE_NEAREST | MF_PHASE_TRANSITIONS | MF_PHASE_EQUILIBRIUM) || !sb->phases)
    return fail(ctx, MF_ERR_INVALID, "phases must be a non-empty set of MF_PHASE_* bits");
  if (sb->flags & ~MF_FLAG_ORIGINAL_PRNG) return fail(ctx, MF_ERR_INVALID, "only MF_FLAG_ORIGINAL_PRNG is accepted");
  if (sb->n_newton < 0 || sb->n_cg < 0) return fail(ctx, MF_ERR_INVALID, "negative solver caps");
  if (!sb->thick_axial || !sb->xb_states || !sb->xb_bound_to || !sb->xb_nearest_bs || !sb->xb_distances ||
      !sb->thin_axial || !sb->tm_states || !sb->thin_bound_to || !sb->keys || !sb->params)
    return fail(ctx, MF_ERR_INVALID, "missing state array");
  const bool dyn = sb->K_lat != nullptr;
  if (dyn && !sb->d_ref) return fail(ctx, MF_ERR_INVALID, "a dynamic lattice spacing needs d_ref with K_lat");
  if ((sb->phases & MF_PHASE_TRANSITIONS) && !(sb->dt > 0.f)) return fail(ctx, MF_ERR_INVALID, "dt must be positive");
  const TopoHost& th = *ctx->topos[sb->topo_id];
  const TopoDev& td = th.dev;
  PopShape ps;
  const PopArgs pa{sb->n_pops, sb->pop_flags, sb->label_stride, sb->pop_params, sb->pop_frac, sb->xb_label,
                   sb->tm_label};
  int rc = check_pops(ctx, pa, {&td}, ps);
  if (rc) return rc;
  CK(cudaSetDevice(ctx->device));
  cudaStream_t st = (cudaStream_t)stream_v;
  // the float32 mode's CTA size (tuned or default), its exact carve
  Cfg c;
  if (!make_cfg(td, th.cfg[0].threads, false, false, dyn, ctx->smem_optin, c, ps))
    return fail(ctx, MF_ERR_INVALID, "lattice and populations exceed shared memory");
  const size_t stride = slot_bytes(td, ps);
  rc = ensure_ws(ctx, stride * (size_t)sb->B);
  if (rc) return rc;
  StepArgs a{};
  a.T = 1;
  a.n_newton = sb->n_newton;
  a.n_cg = sb->n_cg;
  a.flags = (dyn ? FLAG_DYN : 0) | ((sb->flags & MF_FLAG_ORIGINAL_PRNG) ? FLAG_ORIG_PRNG : 0) | c.layout_flags();
  a.resid_warn = INFINITY;
  a.sq64_from = 1 << 20;
  a.u_thin = sb->u_thin;
  a.u_xb = sb->u_xb;
  a.pop = ps;
  StateIO io{};
  io.topo = th.d_struct;
  io.ws = ctx->ws;
  io.ws_stride = stride;
  io.thick_axial = sb->thick_axial;
  io.xb_states = sb->xb_states;
  io.xb_bound = sb->xb_bound_to;
  io.xb_nearest = sb->xb_nearest_bs;
  io.xb_dist = sb->xb_distances;
  io.thin_axial = sb->thin_axial;
  io.tm_states = sb->tm_states;
  io.thin_bound = sb->thin_bound_to;
  io.keys = sb->keys;
  io.params = sb->params;
  io.pCa = sb->pCa;
  io.z = sb->z_line;
  io.ls = sb->lattice_spacing;
  io.K_lat = sb->K_lat;
  io.d_ref = sb->d_ref;
  io.resid_out = sb->residual_out;
  io.ls_out = sb->ls_out;
  io.iters_out = sb->iters_out;
  io.status_out = sb->status_out;
  if (ps.active()) {
    io.pop_params = sb->pop_params;
    io.pop_frac = sb->pop_frac;
    io.xb_label = ps.kx() > 1 ? sb->xb_label : nullptr;
    io.tm_label = ps.kt() > 1 ? sb->tm_label : nullptr;
    io.label_stride = sb->label_stride;
  }
  io.phases = sb->phases;
  io.dt = sb->dt;
  cudaError_t e = launch_state(c.threads, dyn, a, io, sb->B, c.smem_local, st);
  if (e != cudaSuccess) return fail(ctx, MF_ERR_CUDA, "state launch: %s", cudaGetErrorString(e));
  CK(cudaStreamSynchronize(st));
  return MF_OK;
}

int mf_prng_split(uint32_t k0, uint32_t k1, int32_t n, int32_t partitionable, uint32_t* out) {
  if (n < 0 || (!out && n > 0)) return MF_ERR_INVALID;
  for (int i = 0; i < n; ++i) {
    if (partitionable) split_part(k0, k1, (uint32_t)i, out[2 * i], out[2 * i + 1]);
    else split_orig(k0, k1, (uint32_t)n, (uint32_t)i, out[2 * i], out[2 * i + 1]);
  }
  return MF_OK;
}

int mf_prng_uniform(uint32_t k0, uint32_t k1, int32_t n, int32_t partitionable, float* out) {
  if (n < 0 || (!out && n > 0)) return MF_ERR_INVALID;
  for (int i = 0; i < n; ++i) out[i] = bits_to_uniform(bits32(partitionable != 0, k0, k1, (uint32_t)n, (uint32_t)i));
  return MF_OK;
}

}  // extern "C"

#include "mf_server.inc"
