// The fused half-sarcomere timestep: one CTA owns one condition ("slot") and
// advances it through a range of timesteps with every per-condition array
// resident in shared memory.
//
// Per step (reference timestep.py:65-199 inside the scan body of
// simulation.py:679-721):
//   1. rigid thin-filament shift by dz                  simulation.py:683-687
//   2. nearest binding site of every head               kernels/geometry.py:60-262
//   3. tropomyosin Ising transitions + lock             kernels/transitions.py:516-625
//   4. crossbridge transitions + binding bookkeeping    kernels/transitions.py:1081-1245
//   5. Newton-CG equilibrium (fixed or dynamic LS)      kernels/solver.py:329-771
//   6. M-line force and the 52 metrics                  forces.py:588-627, metrics_fn.py:154-417
// Probability tables come from mf_expm.cuh and are rebuilt only when pCa or
// the lattice spacing they were built for changes.
#pragma once
#include "mf_common.cuh"
#include "mf_expm.cuh"

namespace mf {

// Everything one CTA needs to find its condition.  The batched path points
// these into the caller's [B, ...] arrays; the server points them at the
// buffers of a resident slot.
struct CondDesc {
  const TopoDev* topo;
  char* ws;               // resident workspace of this condition (SlotLayout)
  int n_steps;            // total steps of the condition
  int index;              // row in the caller's arrays (test hooks)
  int t0, t1;             // step range of this launch
  int T;                  // stride of z/pCa/ls/metrics rows
  const float* params;    // [44]
  const float* z;         // [T]
  const float* pCa;       // [T]
  const float* ls;        // [T]
  const uint32_t* key;    // [2] key at step 0
  float* metrics;         // [52*T]
  int* status;            // or NULL
  uint32_t* key_out;      // [2] or NULL
  float K_lat, nu, dt;
};

struct StepArgs {
  const CondDesc* cond;
  int T;                 // row stride of the test-hook arrays
  int n_newton, n_cg, flags;
  float resid_warn;
  int sq64_from;         // float64 squaring from this s on (precise mode)
  const float* u_thin;
  const float* u_xb;
  float* x_trace;
  int8_t* st_trace;
  int* bd_trace;
  int max_dof, max_xbs, max_sites;
};

constexpr int FLAG_DYN = 1, FLAG_PRECISE = 2, FLAG_ORIG_PRNG = 4;

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ float warp_min(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ int warp_sum_i(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Shared-memory carve of one condition.
struct Smem {
  float* x;       // [N] node positions (precise mode: displacements)
  float* r;       // [N] residual / CG residual
  float* dx;      // [N] CG solution
  float* pv;      // [N] CG direction
  float* zz;      // [N] preconditioned residual / J p
  float* fxb;     // [X] per-head force or directional term
  float* fdx;     // [X] per-head df/dx at the current Newton point
  float* site;    // [S] per-site crossbridge accumulator (aliases win1 in kinetics)
  int* win2;      // [S] scatter-winner scratch
  float* xb_ax;   // [X] axial offset to the nearest site
  int16_t* xb_bound;
  int16_t* xb_near;
  int16_t* thin_bound;
  int8_t* xb_state;
  int8_t* tm;
  int8_t* tm_new;
  float* cum_tm;  // [27*16]
  float* coef;    // Thomas scan coefficients (thick fwd, thick back, thin fwd, thin back, inv)
  float* scan;    // per-warp scan scratch
  float* P;       // [44]
  float* red;     // reduction scratch [64]
  double* redd;   // [64]
  float* tvec;    // [4*n_thick] titin partials
  float* fdd;     // [X] df/dd per head (dynamic spacing)
  float* frdd;    // [X] d(radial)/dd per head (dynamic spacing)
  int16_t* blist; // [X] heads carrying force this step, increasing index
  int* nbound;    // [1] length of blist
  int* wsum;      // [32] per-warp counts of the compaction scan
  // pre-step (old_state) snapshot read by the metrics epilogue: shared memory
  // when the lattice leaves room, else the resident workspace arrays
  float* old_thick;  // [n_thick*n_crowns]
  int8_t* old_xbs;   // [X]
  int16_t* old_key;  // [X] table row (permissiveness, bin) of the pre-step geometry
  int16_t* xb_key;   // [X] table row used by the latest crossbridge sampling
};

// Thomas coefficient block layout inside coef (floats).
struct CoefLayout {
  int thick_fwd, thick_back, thin_fwd, thin_back, thick_inv, thin_inv, total;
};
__host__ __device__ inline CoefLayout coef_layout(const TopoDev& t) {
  CoefLayout c{};
  int o = 0;
  c.thick_fwd = o; o += t.plan_thick.total;
  c.thick_back = o; o += t.plan_thick.total;
  c.thin_fwd = o; o += t.plan_thin.total;
  c.thin_back = o; o += t.plan_thin.total;
  c.thick_inv = o; o += t.n_crowns;
  c.thin_inv = o; o += t.n_sites;
  c.total = (o + 3) / 4 * 4;
  return c;
}

template <int NT>
struct Sim {
  static constexpr int NW = NT / 32;
  const TopoDev& T;
  const StepArgs& A;
  Smem s;
  CoefLayout cl;
  SlotLayout L;
  char* ws;
  int b;        // caller row
  int tid, lane, warp;
  bool dyn, precise, part;
  float Kl, nu_c, dtm;
  double zref;  // precise mode thin reference z
  float dvar;   // lattice spacing unknown (dynamic) / fixed spacing
  float d_ref;
  int status;
  int Tstride;
  int redbuf = 0;

  __device__ Sim(const TopoDev& t, const StepArgs& a) : T(t), A(a) {}

  // ------------------------------------------------------------------
  // reductions
  // ------------------------------------------------------------------
  __device__ float bsum(float v) {
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) s.red[warp] = v;
    __syncthreads();
    float t = 0.f;
    for (int w = 0; w < NW; ++w) t += s.red[w];
    return t;
  }
  __device__ double bsum_d(double v) {
    v = warp_sum_d(v);
    __syncthreads();
    if (lane == 0) s.redd[warp] = v;
    __syncthreads();
    double t = 0.0;
    for (int w = 0; w < NW; ++w) t += s.redd[w];
    return t;
  }
  __device__ float bmax(float v) {
    v = warp_max(v);
    __syncthreads();
    if (lane == 0) s.red[warp] = v;
    __syncthreads();
    float t = s.red[0];
    for (int w = 1; w < NW; ++w) t = fmaxf(t, s.red[w]);
    return t;
  }
  __device__ float bmin(float v) {
    v = warp_min(v);
    __syncthreads();
    if (lane == 0) s.red[warp] = v;
    __syncthreads();
    float t = s.red[0];
    for (int w = 1; w < NW; ++w) t = fminf(t, s.red[w]);
    return t;
  }
  // K floats at once: entries k < nmax reduced with max, the rest summed
  template <int K>
  __device__ void bred(float (&v)[K], int nmax) {
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = k < nmax ? warp_max(v[k]) : warp_sum(v[k]);
    __syncthreads();
    if (lane == 0)
#pragma unroll
      for (int k = 0; k < K; ++k) s.red[k * NW + warp] = v[k];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; ++k) {
      float t = s.red[k * NW];
      for (int w = 1; w < NW; ++w) t = k < nmax ? fmaxf(t, s.red[k * NW + w]) : t + s.red[k * NW + w];
      v[k] = t;
    }
  }
  // sum of K floats at once
  template <int K>
  __device__ void bsum_k(float (&v)[K]) {
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = warp_sum(v[k]);
    __syncthreads();
    if (lane == 0)
#pragma unroll
      for (int k = 0; k < K; ++k) s.red[k * NW + warp] = v[k];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; ++k) {
      float t = 0.f;
      for (int w = 0; w < NW; ++w) t += s.red[k * NW + w];
      v[k] = t;
    }
  }
  template <int K>
  __device__ void bsum_ki(int (&v)[K]) {
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = warp_sum_i(v[k]);
    __syncthreads();
    int* ri = reinterpret_cast<int*>(s.red);
    if (lane == 0)
#pragma unroll
      for (int k = 0; k < K; ++k) ri[k * NW + warp] = v[k];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; ++k) {
      int t = 0;
      for (int w = 0; w < NW; ++w) t += ri[k * NW + w];
      v[k] = t;
    }
  }

  // ------------------------------------------------------------------
  // geometry helpers
  // ------------------------------------------------------------------
  __device__ __forceinline__ int crown_node(int xb) const { return xb / T.nxb; }
  __device__ __forceinline__ int thin_of(int xb) const { return T.xb_face[xb] / 3; }
  // absolute site position (double; precise mode reconstructs from zref)
  __device__ __forceinline__ double site_pos_d(int gsite) const {
    const float u = s.x[T.n_thick_nodes + gsite];
    return precise ? (zref - (double)T.bind_off[gsite]) + (double)u : (double)u;
  }
  __device__ __forceinline__ double crown_pos_d(int node) const {
    const float u = s.x[node];
    return precise ? (double)T.crown_off[node] + (double)u : (double)u;
  }
  // axial offset site - crown (float)
  __device__ __forceinline__ float xb_offset(int gsite, int node) const {
    if (!precise) return s.x[T.n_thick_nodes + gsite] - s.x[node];
    const float G = (float)((zref - (double)T.bind_off[gsite]) - (double)T.crown_off[node]);
    return G + (s.x[T.n_thick_nodes + gsite] - s.x[node]);
  }
  // z - x_last of thick filament t
  __device__ __forceinline__ float titin_ad(int t, float zl) const {
    const int node = t * T.n_crowns + T.n_crowns - 1;
    if (!precise) return zl - s.x[node];
    return (float)((double)zl - (double)T.crown_off[node]) - s.x[node];
  }

  // ------------------------------------------------------------------
  // Thomas preconditioner: per-filament affine scans in JAX association order
  // ------------------------------------------------------------------
  __device__ void scan_b(const ScanPlan& pl, const float* Acoef, float* buf) {
    // buf[0..n) holds b of level 0; levels above are built in place.
    for (int l = 0; l + 1 < pl.levels; ++l) {
      const int nn = pl.len[l + 1];
      const float* Al = Acoef + pl.off[l];
      const float* El = buf + pl.off[l];
      float* En = buf + pl.off[l + 1];
      for (int k = lane; k < nn; k += 32) En[k] = fmaf(Al[2 * k + 1], El[2 * k], El[2 * k + 1]);
      __syncwarp();
    }
    for (int l = pl.levels - 2; l >= 0; --l) {
      const int nl = pl.len[l], nn = pl.len[l + 1];
      const float* Al = Acoef + pl.off[l];
      float* El = buf + pl.off[l];
      const float* Sn = buf + pl.off[l + 1];
      for (int k = lane; 2 * k < nl; k += 32) {
        if (k >= 1) El[2 * k] = fmaf(Al[2 * k], Sn[k - 1], El[2 * k]);
        if (k < nn) El[2 * k + 1] = Sn[k];
      }
      __syncwarp();
    }
  }

  // Node ownership: warp w owns filaments w, w + NW, ...; lane l handles
  // nodes l, l + 32, ... of each.  Every elementwise vector update and the
  // Thomas solves stay inside a warp, so only the crossbridge coupling and
  // the dot products need block barriers.
  template <class Fn>
  __device__ __forceinline__ void own_nodes(Fn&& fn) const {
    const int nf = T.n_thick + T.n_thin;
    for (int f = warp; f < nf; f += NW) {
      const bool thick = f < T.n_thick;
      const int n = thick ? T.n_crowns : T.n_sites;
      const int base = thick ? f * T.n_crowns : T.n_thick_nodes + (f - T.n_thick) * T.n_sites;
      for (int j = lane; j < n; j += 32) fn(base + j, f, j, thick);
    }
  }

  // Thomas substitutions of one filament as warp-shuffle affine scans: lane l
  // owns nodes [l*E, l*E+E); a local scan per lane, a 5-step Kogge-Stone
  // composition across lanes, then the lane's own nodes.  Same result as the
  // tree order in exact arithmetic; used in precise mode, where the
  // reference's float32 association order is not the target.
  template <int E>
  __device__ __forceinline__ void thomas_shfl(const float* in, float* out, int n, const float* Af,
                                              const float* Ab, const float* inv) {
    float y[E], a[E];
    const int i0 = lane * E;
    // forward: y[i] = a_f[i] * y[i-1] + r[i], y[-1] = 0
    float A = 1.f, Bv = 0.f;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int i = i0 + e;
      const bool ok = i < n;
      a[e] = ok ? Af[i] : 1.f;
      y[e] = ok ? in[i] : 0.f;
      Bv = fmaf(a[e], Bv, y[e]);
      A = a[e] * A;
    }
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const float Ap = __shfl_up_sync(0xffffffffu, A, o), Bp = __shfl_up_sync(0xffffffffu, Bv, o);
      if (lane >= o) {
        Bv = fmaf(A, Bp, Bv);
        A = A * Ap;
      }
    }
    float yp = __shfl_up_sync(0xffffffffu, Bv, 1);
    if (lane == 0) yp = 0.f;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      yp = fmaf(a[e], yp, y[e]);
      y[e] = yp;
    }
    // backward: x[i] = (y[i] * inv[i]) + a_b[i] * x[i+1], x[n] = 0
    A = 1.f;
    Bv = 0.f;
#pragma unroll
    for (int e = E - 1; e >= 0; --e) {
      const int i = i0 + e;
      const bool ok = i < n;
      a[e] = ok ? Ab[n - 1 - i] : 1.f;
      y[e] = ok ? y[e] * inv[i] : 0.f;
      Bv = fmaf(a[e], Bv, y[e]);
      A = a[e] * A;
    }
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const float Ap = __shfl_down_sync(0xffffffffu, A, o), Bp = __shfl_down_sync(0xffffffffu, Bv, o);
      if (lane + o < 32) {
        Bv = fmaf(A, Bp, Bv);
        A = A * Ap;
      }
    }
    float xp = __shfl_down_sync(0xffffffffu, Bv, 1);
    if (lane == 31) xp = 0.f;
#pragma unroll
    for (int e = E - 1; e >= 0; --e) {
      xp = fmaf(a[e], xp, y[e]);
      const int i = i0 + e;
      if (i < n) out[i] = xp;
    }
  }

  // out = M^{-1} in on this warp's own filaments (no block barrier needed).
  __device__ void precondition_own(const float* in, float* out) {
    const int nf = T.n_thick + T.n_thin;
    if (precise) {
      __syncwarp();
      for (int f = warp; f < nf; f += NW) {
        const bool thick = f < T.n_thick;
        const int n = thick ? T.n_crowns : T.n_sites;
        const int base = thick ? f * T.n_crowns : T.n_thick_nodes + (f - T.n_thick) * T.n_sites;
        const float* Af = s.coef + (thick ? cl.thick_fwd : cl.thin_fwd);
        const float* Ab = s.coef + (thick ? cl.thick_back : cl.thin_back);
        const float* inv = s.coef + (thick ? cl.thick_inv : cl.thin_inv);
        if (n <= 64) thomas_shfl<2>(in + base, out + base, n, Af, Ab, inv);
        else if (n <= 96) thomas_shfl<3>(in + base, out + base, n, Af, Ab, inv);
        else thomas_shfl<4>(in + base, out + base, n, Af, Ab, inv);
      }
      __syncwarp();
      return;
    }
    float* buf = s.scan + warp * (T.plan_thin.total > T.plan_thick.total ? T.plan_thin.total
                                                                          : T.plan_thick.total);
    __syncwarp();
    for (int f = warp; f < nf; f += NW) {
      const bool thick = f < T.n_thick;
      const int n = thick ? T.n_crowns : T.n_sites;
      const int base = thick ? f * T.n_crowns : T.n_thick_nodes + (f - T.n_thick) * T.n_sites;
      const ScanPlan& pl = thick ? T.plan_thick : T.plan_thin;
      const float* Af = s.coef + (thick ? cl.thick_fwd : cl.thin_fwd);
      const float* Ab = s.coef + (thick ? cl.thick_back : cl.thin_back);
      const float* inv = s.coef + (thick ? cl.thick_inv : cl.thin_inv);
      for (int i = lane; i < n; i += 32) buf[i] = in[base + i];
      __syncwarp();
      scan_b(pl, Af, buf);
      // back substitution input: (y * inv) reversed
      float tmp[4];
      int cnt = 0;
      for (int i = lane; i < n; i += 32) tmp[cnt++] = buf[i] * inv[i];
      __syncwarp();
      cnt = 0;
      for (int i = lane; i < n; i += 32) buf[n - 1 - i] = tmp[cnt++];
      __syncwarp();
      scan_b(pl, Ab, buf);
      for (int i = lane; i < n; i += 32) out[base + i] = buf[n - 1 - i];
      __syncwarp();
    }
  }

  // One-barrier block reduction of K floats (sum) with an optional max in
  // slot 0; double-buffered so consecutive reductions need no extra barrier.
  template <int K>
  __device__ __forceinline__ void reduce(float (&v)[K], bool max0) {
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = (max0 && k == 0) ? warp_max(v[k]) : warp_sum(v[k]);
    float* rb = s.red + 1024 + redbuf * 96;  // clear of bred/bsum_* (red[0, 1024)) and red[1535]
    redbuf ^= 1;
    if (lane == 0)
#pragma unroll
      for (int k = 0; k < K; ++k) rb[k * NW + warp] = v[k];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; ++k) {
      float t = rb[k * NW];
      for (int w = 1; w < NW; ++w) t = (max0 && k == 0) ? fmaxf(t, rb[k * NW + w]) : t + rb[k * NW + w];
      v[k] = t;
    }
  }

  // Factor the negated backbone matrices and precompute the a-components of
  // every scan node (solver.py:128-162, 165-219, 243-282); once per condition.
  __device__ void build_precond_coef(float* coef_g) {
    if (tid < 2) {
      const bool thick = tid == 0;
      const int n = thick ? T.n_crowns : T.n_sites;
      const float k = thick ? s.P[THICK_K] : s.P[THIN_K];
      const ScanPlan& pl = thick ? T.plan_thick : T.plan_thin;
      float* Af = coef_g + (thick ? cl.thick_fwd : cl.thin_fwd);
      float* Ab = coef_g + (thick ? cl.thick_back : cl.thin_back);
      float* inv = coef_g + (thick ? cl.thick_inv : cl.thin_inv);
      // diag (negated): 2k + 1e-9, boundary k + 1e-9 (thick: last, thin: first)
      const float off = -k;  // negated off-diagonals
      float md_prev = 0.f;
      for (int i = 0; i < n; ++i) {
        const bool bnd = thick ? (i == n - 1) : (i == 0);
        const float diag = -((bnd ? -1.0f : -2.0f) * k) + 1e-9f;
        float md;
        if (i == 0) {
          md = diag;
          Af[0] = 1.0f;
        } else {
          const float m = off / md_prev;
          md = diag - m * off;
          Af[i] = -m;
        }
        inv[i] = 1.0f / md;
        md_prev = md;
      }
      // back-substitution a's: a_back[i] = -upper[i]*inv[i] (i<n-1), a_back[n-1]=0; reversed
      for (int j = 0; j < n; ++j) {
        const int i = n - 1 - j;
        Ab[j] = (i < n - 1) ? (-off) * inv[i] : 0.0f;
      }
      // a-components of the down-sweep tree: A_{l+1}[k] = A_l[2k+1] * A_l[2k]
      for (int pass = 0; pass < 2; ++pass) {
        float* Ac = pass == 0 ? Af : Ab;
        for (int l = 0; l + 1 < pl.levels; ++l)
          for (int kk = 0; kk < pl.len[l + 1]; ++kk)
            Ac[pl.off[l + 1] + kk] = Ac[pl.off[l] + 2 * kk + 1] * Ac[pl.off[l] + 2 * kk];
      }
    }
  }

  // ------------------------------------------------------------------
  // forces
  // ------------------------------------------------------------------
  // Per-head force f, df/dx and (dynamic) df/dd, dfr/dd, fr at spacing d.
  __device__ __forceinline__ void xb_force(int xb, float d, float& f, float& fx, float& fd,
                                           float& frd, float& fr) const {
    const int st = s.xb_state[xb];
    const int bnd = s.xb_bound[xb];
    f = fx = fd = frd = fr = 0.f;
    if (st < 1 || st > 3 || bnd < 0) return;
    const bool strong = st >= 2;
    const float gk = strong ? s.P[XB_G_K_STRONG] : s.P[XB_G_K_WEAK];
    const float g0 = strong ? s.P[XB_G_REST_STRONG] : s.P[XB_G_REST_WEAK];
    const float ck = strong ? s.P[XB_C_K_STRONG] : s.P[XB_C_K_WEAK];
    const float c0 = strong ? s.P[XB_C_REST_STRONG] : s.P[XB_C_REST_WEAK];
    const int gs = thin_of(xb) * T.n_sites + bnd;
    const float x = xb_offset(gs, crown_node(xb));
    const float r = sqrtf(x * x + d * d);
    const float rs = r > 1e-10f ? r : 1e-10f;
    const float cs = x / rs, sn = d / rs;
    const float th = atan2f(d, x);
    const float dth = th - c0;
    f = gk * (r - g0) * cs - (1.0f / rs) * ck * dth * sn;
    const float ir2 = 1.0f / (r * r);
    fx = gk * (cs * cs + (1.0f - g0 / r) * sn * sn) + ck * ir2 * (2.0f * dth * sn * cs + sn * sn);
    if (dyn) {
      fd = gk * sn * cs * (g0 / r) - ck * ir2 * (sn * cs + dth * (cs * cs - sn * sn));
      frd = gk * (sn * sn + (r - g0) * cs * cs / r) + ck * ir2 * (cs * cs - 2.0f * dth * sn * cs);
      fr = gk * (r - g0) * sn + (1.0f / rs) * ck * dth * cs;
    }
  }

  // titin: force terms at the last crown of thick t (forces.py:130-150)
  __device__ __forceinline__ void titin(int t, float zl, float d, float& ax, float& a_x, float& a_d,
                                        float& r_d, float& rad) const {
    const float ad = titin_ad(t, zl);
    const float Lt = sqrtf(ad * ad + d * d);
    float arg = s.P[TITIN_B] * (Lt - s.P[TITIN_REST]);
    const bool clipped = arg < -100.f || arg > 100.f;
    arg = fminf(fmaxf(arg, -100.f), 100.f);
    const float Ft = fmaxf(s.P[TITIN_A] * expf(arg), 0.f);
    const float cosang = Lt > 0.f ? ad / Lt : 0.f;
    ax = 6.0f * (Ft * cosang);
    const float bb = clipped ? 0.f : s.P[TITIN_B];
    const float L2 = Lt * Lt, L3 = L2 * Lt;
    a_x = -6.0f * Ft * (bb * ad * ad / L2 + d * d / L3);
    a_d = 6.0f * Ft * ad * d * (bb / L2 - 1.0f / L3);
    r_d = 6.0f * Ft * (bb * d * d / L2 + ad * ad / L3);
    const float Ls = Lt > 1e-10f ? Lt : 1e-10f;
    rad = 6.0f * Ft * (d / Ls);
  }

  // Compact list of the heads that carry force this step (states 1-3 with a
  // site), in increasing head index (block prefix scan, deterministic), plus
  // the number of heads on every site.  Clears the per-head and per-site
  // accumulators.  Sites holding 3+ heads are summed in head order by their
  // node owner (sums of two are order-free; the reference adds in index
  // order, transitions/forces.py segment_sum).
  __device__ void build_bound_list() {
    const int X = T.total_xbs, S = T.n_sites_total;
    int* cnt = s.win2;
    __syncthreads();
    for (int g = tid; g < S; g += NT) {
      s.site[g] = 0.f;
      cnt[g] = 0;
    }
    __syncthreads();
    int base = 0;
    for (int c = 0; c < X; c += NT) {
      const int i = c + tid;
      bool f = false;
      if (i < X) {
        s.fxb[i] = 0.f;
        const int st = s.xb_state[i];
        f = st >= 1 && st <= 3 && s.xb_bound[i] >= 0;
        if (f) atomicAdd(&cnt[thin_of(i) * T.n_sites + s.xb_bound[i]], 1);
      }
      const unsigned m = __ballot_sync(0xffffffffu, f);
      if (lane == 0) s.wsum[warp] = __popc(m);
      __syncthreads();
      int off = base, tot = 0;
      for (int w = 0; w < NW; ++w) {
        const int v = s.wsum[w];
        off += w < warp ? v : 0;
        tot += v;
      }
      if (f) s.blist[off + __popc(m & ((1u << lane) - 1u))] = (int16_t)i;
      base += tot;
      __syncthreads();
    }
    if (tid == 0) *s.nbound = base;
    __syncthreads();
  }

  // crossbridge sum of a site with 3+ bound heads: -sum of fxb in head order
  __device__ float ordered_site_sum(int g) const {
    const int nb = *s.nbound;
    float acc = 0.f;
    int prev = -1;
    while (true) {
      int nxt = 0x7fffffff;
      for (int k = 0; k < nb; ++k) {
        const int i = s.blist[k];
        if (i > prev && i < nxt && thin_of(i) * T.n_sites + s.xb_bound[i] == g) nxt = i;
      }
      if (nxt == 0x7fffffff) break;
      acc = acc + (-s.fxb[nxt]);
      prev = nxt;
    }
    return acc;
  }

  // Residual F(x) into s.r (own nodes); caches df/dx per bound head and the
  // titin partials for the JVPs of the next Newton iteration.  Returns max|F|
  // over the augmented vector; *frad = radial residual, *jdd = dF_rad/dd.
  // In precise mode the node forces are accumulated in float64.
  __device__ float residual(float zl, float d, float* frad, float* jdd, int bad_in, int* bad_out) {
    const int nb = *s.nbound;
    float rad_part = 0.f, jdd_part = 0.f;
    const int any_bad = __syncthreads_or(bad_in);
    if (bad_out) *bad_out = any_bad;
    for (int k = tid; k < nb; k += NT) {
      const int i = s.blist[k];
      float f, fx, fd, frd, fr;
      xb_force(i, d, f, fx, fd, frd, fr);
      s.fxb[i] = f;
      s.fdx[i] = fx;
      if (dyn) {
        s.fdd[i] = fd;
        s.frdd[i] = frd;
        rad_part += fr;
        jdd_part += frd;
      }
      const int gs = thin_of(i) * T.n_sites + s.xb_bound[i];
      if (s.win2[gs] < 3) atomicAdd(&s.site[gs], -f);
    }
    if (tid < T.n_thick) {
      float ax, a_x, a_d, r_d, rad;
      titin(tid, zl, d, ax, a_x, a_d, r_d, rad);
      s.tvec[tid] = ax;
      s.tvec[T.n_thick + tid] = a_x;
      s.tvec[2 * T.n_thick + tid] = a_d;
      s.tvec[3 * T.n_thick + tid] = r_d;
      if (dyn) {
        rad_part += rad;
        jdd_part += r_d;
      }
    }
    __syncthreads();
    const float kth = s.P[THICK_K], ktn = s.P[THIN_K];
    float fmax = 0.f;
    own_nodes([&](int i, int f, int j, bool thick) {
      double F;
      if (thick) {
        const int c = j;
        float xsum = s.fxb[i * T.nxb];
        for (int q = 1; q < T.nxb; ++q) xsum += s.fxb[i * T.nxb + q];
        if (!precise) {
          const float xm = c > 0 ? s.x[i - 1] : 0.f;
          const float sp_c = ((s.x[i] - xm) - T.crown_rest[i]) * kth;
          const float sp_n = (c + 1 < T.n_crowns) ? ((s.x[i + 1] - s.x[i]) - T.crown_rest[i + 1]) * kth : s.tvec[f];
          F = (double)((sp_n - sp_c) + xsum);
        } else {
          const double um = c > 0 ? (double)s.x[i - 1] : 0.0;
          const double e_c = ((double)s.x[i] - um) + (double)T.thick_c[i];
          const double spn = (c + 1 < T.n_crowns)
                                 ? (((double)s.x[i + 1] - (double)s.x[i]) + (double)T.thick_c[i + 1]) * (double)kth
                                 : (double)s.tvec[f];
          F = (spn - e_c * (double)kth) + (double)xsum;
        }
      } else {
        const int g = i - T.n_thick_nodes;
        const float acc = s.win2[g] < 3 ? s.site[g] : ordered_site_sum(g);
        s.site[g] = 0.f;
        if (!precise) {
          const float xn = (j + 1 < T.n_sites) ? s.x[i + 1] : zl;
          const float sp_j = ((xn - s.x[i]) - T.bind_rest[g]) * ktn;
          const float sp_m = j > 0 ? ((s.x[i] - s.x[i - 1]) - T.bind_rest[g - 1]) * ktn : 0.f;
          F = (double)((sp_j - sp_m) + acc);
        } else {
          const double un = (j + 1 < T.n_sites) ? (double)s.x[i + 1] : 0.0;
          double e_j = (un - (double)s.x[i]) + (double)T.thin_c[g];
          if (j + 1 == T.n_sites) e_j += (double)zl - zref;  // anchor vs reference z
          const double e_m = j > 0 ? ((double)s.x[i] - (double)s.x[i - 1]) + (double)T.thin_c[g - 1] : 0.0;
          F = (e_j - e_m) * (double)ktn + (double)acc;
        }
      }
      s.r[i] = (float)F;
      fmax = fmaxf(fmax, (float)fabs(F));
    });
    float v[3] = {fmax, rad_part, jdd_part};
    reduce<3>(v, true);
    float m = v[0];
    if (dyn) {
      const float Fr = -Kl * (d - d_ref) + (-v[1]);
      *frad = Fr;
      m = fmaxf(m, fabsf(Fr));
      if (jdd) *jdd = -Kl - v[2];
    }
    return m;
  }

  // out = -(J [v, vd]) on own nodes; returns the augmented dot(v, out), *out_d
  // the radial component.
  __device__ float neg_jvp(const float* v, float vd, float* out, float* out_d) {
    const int nb = *s.nbound;
    float rad_part = 0.f;
    __syncthreads();  // v complete
    for (int k = tid; k < nb; k += NT) {
      const int i = s.blist[k];
      const int gs = thin_of(i) * T.n_sites + s.xb_bound[i];
      const float dxd = v[T.n_thick_nodes + gs] - v[crown_node(i)];
      float w = s.fdx[i] * dxd;
      if (dyn) {
        w = w + s.fdd[i] * vd;
        rad_part += -(s.fdd[i] * dxd) - s.frdd[i] * vd;
      }
      s.fxb[i] = w;
      if (s.win2[gs] < 3) atomicAdd(&s.site[gs], -w);
    }
    if (dyn && tid < T.n_thick) {
      const int last = tid * T.n_crowns + T.n_crowns - 1;
      rad_part += s.tvec[2 * T.n_thick + tid] * v[last] - s.tvec[3 * T.n_thick + tid] * vd;
    }
    __syncthreads();
    const float kth = s.P[THICK_K], ktn = s.P[THIN_K];
    float dot = 0.f;
    own_nodes([&](int i, int f, int j, bool thick) {
      float J;
      if (thick) {
        const float vm = j > 0 ? v[i - 1] : 0.f;
        const float sc = (v[i] - vm) * kth;
        float sn;
        if (j + 1 < T.n_crowns) sn = (v[i + 1] - v[i]) * kth;
        else {
          sn = s.tvec[T.n_thick + f] * v[i];
          if (dyn) sn = sn + s.tvec[2 * T.n_thick + f] * vd;
        }
        float xs = s.fxb[i * T.nxb];
        for (int q = 1; q < T.nxb; ++q) xs += s.fxb[i * T.nxb + q];
        J = (sn - sc) + xs;
      } else {
        const int g = i - T.n_thick_nodes;
        const float vn = (j + 1 < T.n_sites) ? v[i + 1] : 0.f;
        const float sj = (vn - v[i]) * ktn;
        const float sm = j > 0 ? (v[i] - v[i - 1]) * ktn : 0.f;
        J = (sj - sm) + (s.win2[g] < 3 ? s.site[g] : ordered_site_sum(g));
        s.site[g] = 0.f;
      }
      const float o = -J;
      out[i] = o;
      dot = fmaf(v[i], o, dot);
    });
    float r2[2] = {dot, rad_part};
    reduce<2>(r2, false);
    if (dyn) {
      const float od = -(r2[1] + (-Kl) * vd);
      *out_d = od;
      return r2[0] + vd * od;
    }
    return r2[0];
  }

  // ------------------------------------------------------------------
  // Newton-CG (solver.py:329-427, 599-656)
  // ------------------------------------------------------------------
  __device__ void solve(float zl, float& d, double& resid, int& iters, bool dyn_jdd) {
    const float tol = fmaxf(s.P[SOLVER_TOL], fmaxf(s.P[THICK_K] * 1e-4f, 0.25f));
    float frad = 0.f, jdd = 0.f;
    float fmx = residual(zl, d, &frad, &jdd, 0, nullptr);
    // exact radial diagonal at the pre-solve point (solver.py:633-638)
    const float J_dd_inv = dyn_jdd ? -1.0f / jdd : 0.f;
    int it = 0, bad = 0;
    while (fmx > tol && it < A.n_newton) {
      float r_d = frad, z_d = 0.f, p_d = 0.f, dx_d = 0.f, Ap_d = 0.f;
      precondition_own(s.r, s.zz);
      float part[1] = {0.f};
      own_nodes([&](int i, int, int, bool) {
        s.pv[i] = s.zz[i];
        s.dx[i] = A.n_cg == 0 ? s.zz[i] : 0.f;
        part[0] = fmaf(s.r[i], s.zz[i], part[0]);
      });
      if (dyn) {
        z_d = J_dd_inv * r_d;
        p_d = z_d;
        if (A.n_cg == 0) dx_d = z_d;
      }
      reduce<1>(part, false);
      float rz = part[0] + (dyn ? r_d * z_d : 0.f);
      for (int k = 0; k < A.n_cg; ++k) {
        const float pAp = neg_jvp(s.pv, p_d, s.zz, &Ap_d);
        const float alpha = rz / (pAp + 1e-30f);
        own_nodes([&](int i, int, int, bool) {
          s.dx[i] = fmaf(alpha, s.pv[i], s.dx[i]);
          s.r[i] = s.r[i] - alpha * s.zz[i];
        });
        dx_d = fmaf(alpha, p_d, dx_d);
        r_d = r_d - alpha * Ap_d;
        precondition_own(s.r, s.zz);
        float rzp[1] = {0.f};
        own_nodes([&](int i, int, int, bool) { rzp[0] = fmaf(s.r[i], s.zz[i], rzp[0]); });
        if (dyn) z_d = J_dd_inv * r_d;
        reduce<1>(rzp, false);
        const float rz_new = rzp[0] + (dyn ? r_d * z_d : 0.f);
        const float beta = rz_new / (rz + 1e-30f);
        own_nodes([&](int i, int, int, bool) { s.pv[i] = fmaf(beta, s.pv[i], s.zz[i]); });
        p_d = fmaf(beta, p_d, z_d);
        rz = rz_new;
      }
      // x += dx with non-finite entries zeroed
      int bad_local = 0;
      own_nodes([&](int i, int, int, bool) {
        float v = s.dx[i];
        if (!isfinite(v)) { v = 0.f; bad_local = 1; }
        s.x[i] = s.x[i] + v;
      });
      if (dyn) {
        float v = dx_d;
        if (!isfinite(v)) v = 0.f;
        d = fmaxf(d + v, 1.0f);
      }
      fmx = residual(zl, d, &frad, nullptr, bad_local, &bad);
      if (bad) status |= MF_NONFINITE_BIT;
      ++it;
    }
    resid = fmx;
    iters = it;
    if (!isfinite(fmx)) status |= MF_NONFINITE_BIT;
  }
  static constexpr int MF_NONFINITE_BIT = 1;

  // ------------------------------------------------------------------
  // probability tables (built when (pCa, d) differ from the cached key)
  // ------------------------------------------------------------------
  __device__ void build_tables(float pCa, float d, bool sampling, bool absorbing) {
    float* cum_xb = reinterpret_cast<float*>(ws + L.cum_xb);
    float* pabs = reinterpret_cast<float*>(ws + L.pabs);
    const int nb = T.n_bins;
    const int sq64 = A.sq64_from;
    if (sampling) {
      for (int m = tid; m < 27; m += NT) {
        float Q[16];
        tm_generator(s.P, pCa, m, Q);
        for (int i = 0; i < 16; ++i) Q[i] = Q[i] * dtm;
        expm_pade6<4>(Q, sq64);
        for (int r = 0; r < 4; ++r) cum4(Q + 4 * r, s.cum_tm + m * 16 + 4 * r);
      }
    }
    const int nwork = (sampling ? 2 * nb : 0) + (absorbing ? 2 * nb : 0);
    for (int w = tid; w < nwork; w += NT) {
      const bool is_abs = !sampling || w >= 2 * nb;
      const int key = is_abs && sampling ? w - 2 * nb : w;
      const int bin = key % nb;
      const float perm = key >= nb ? 1.0f : 0.0f;
      float Q[36];
      xb_generator(s.P, pCa, T.centers[bin], d, perm, Q);
      if (is_abs)
        for (int j = 0; j < 6; ++j) { Q[24 + j] = 0.f; Q[j] = 0.f; }
      for (int i = 0; i < 36; ++i) Q[i] = Q[i] * dtm;
      expm_pade6<6>(Q, sq64);
      if (is_abs) {
        pabs[key * 3 + 0] = Q[3 * 6 + 4];  // P_abs[3,4]
        pabs[key * 3 + 1] = Q[2 * 6 + 0];  // P_abs[2,0]
        pabs[key * 3 + 2] = Q[3 * 6 + 0];  // P_abs[3,0]
      } else {
        for (int r = 0; r < 6; ++r) cum6(Q + 6 * r, cum_xb + key * 36 + 6 * r);
      }
    }
  }

  // ------------------------------------------------------------------
  // kinetics
  // ------------------------------------------------------------------
  __device__ void nearest(float d) {
    const int X = T.total_xbs;
    for (int i = tid; i < X; i += NT) {
      const int face = T.xb_face[i];
      const int thin = face / 3;
      const int node = crown_node(i);
      const int nv = T.face_n[face];
      const int16_t* cand = T.face_sites + face * T.width;
      int bestk = 0;
      if (!precise) {
        const float head = s.x[node] + 13.0f;
        float best = INFINITY;
        for (int k = 0; k < T.width; ++k) {
          const float pos = s.x[T.n_thick_nodes + thin * T.n_sites + cand[k]];
          if (k < nv && pos > 0.0f) {
            const float dist = fabsf(pos - head);
            if (dist < best) { best = dist; bestk = k; }
          }
        }
      } else {
        const double head = crown_pos_d(node) + 13.0;
        double best = INFINITY;
        for (int k = 0; k < T.width; ++k) {
          const double pos = site_pos_d(thin * T.n_sites + cand[k]);
          if (k < nv && pos > 0.0) {
            const double dist = fabs(pos - head);
            if (dist < best) { best = dist; bestk = k; }
          }
        }
      }
      const int site = cand[bestk];
      s.xb_near[i] = (int16_t)site;
      s.xb_ax[i] = xb_offset(thin * T.n_sites + site, node);
    }
    (void)d;
  }

  __device__ __forceinline__ float uniform_of(const uint32_t* key, int n, int i, const float* inj,
                                              size_t inj_off) const {
    if (inj) return inj[inj_off + i];
    return bits_to_uniform(bits32(part, key[0], key[1], (uint32_t)n, (uint32_t)i));
  }

  __device__ void thin_step(const uint32_t* sub, size_t inj_off) {
    const int S = T.n_sites_total;
    for (int g = tid; g < S; g += NT) {
      const int t = g / T.n_sites;
      const int j = g % T.n_sites;
      const int pj = T.tm_prev[g], nj = T.tm_next[g];
      const int sp = s.tm[t * T.n_sites + pj], sn = s.tm[t * T.n_sites + nj];
      const bool pr = pj != j, nr = nj != j;
      const int n2 = (pr && sp == 2) + (nr && sn == 2);
      const int n3 = (pr && sp == 3) + (nr && sn == 3);
      const int nc = (pr && sp <= 1) + (nr && sn <= 1);
      const int cfg = n2 * 9 + n3 * 3 + nc;
      const int st = s.tm[g];
      const float u = uniform_of(sub, S, g, A.u_thin, inj_off);
      int ns = 0;
      if (st == 3 && s.thin_bound[g] >= 0) {
        // locked row [0,0,0,1]: first cumsum entry above u is index 3
        ns = u < 0.f ? 0 : (u < 1.0f ? 3 : 0);
      } else {
        const float* c = s.cum_tm + cfg * 16 + st * 4;
        ns = u < c[0] ? 0 : (u < c[1] ? 1 : (u < c[2] ? 2 : (u < c[3] ? 3 : 0)));
      }
      s.tm_new[g] = (int8_t)ns;
    }
    __syncthreads();
    for (int g = tid; g < S; g += NT) s.tm[g] = s.tm_new[g];
    __syncthreads();
  }

  __device__ __forceinline__ int bin_of(float x) const {
    // clip(digitize(x, edges) - 1, 0, n_bins - 1); digitize = #edges <= x
    const int nb = T.n_bins;
    const float lo = T.edges[0], hi = T.edges[nb];
    float kf = floorf((x - lo) * ((float)nb / (hi - lo)));
    kf = fminf(fmaxf(kf, 0.0f), (float)nb);
    int k = (int)kf;
    while (k > 0 && T.edges[k] > x) --k;
    while (k < nb && T.edges[k + 1] <= x) ++k;
    // now edges[k] <= x < edges[k+1] (or x below edges[0] -> k = 0 with edges[0] > x)
    int dg = (x >= T.edges[0]) ? k + 1 : 0;  // number of edges <= x
    if (x != x) dg = nb + 1;                  // NaN: digitize puts it past the last edge
    int bin = dg - 1;
    return bin < 0 ? 0 : (bin > nb - 1 ? nb - 1 : bin);
  }

  __device__ void thick_step(const uint32_t* sub, size_t inj_off) {
    const int X = T.total_xbs, S = T.n_sites_total;
    const float* cum_xb = reinterpret_cast<const float*>(ws + L.cum_xb);
    int* win1 = reinterpret_cast<int*>(s.site);
    for (int g = tid; g < S; g += NT) { win1[g] = -1; s.win2[g] = -1; }
    __syncthreads();
    // sample, decide binding, and bid for the two scatter targets
    for (int i = tid; i < X; i += NT) {
      const int thin = thin_of(i);
      const int near = s.xb_near[i];
      const int site = near < 0 ? 0 : (near > T.n_sites - 1 ? T.n_sites - 1 : near);
      const int tgt = thin * T.n_sites + site;
      const bool perm = (s.tm[tgt] == 3) && T.xb_valid[i];
      const int key = (perm ? T.n_bins : 0) + bin_of(s.xb_ax[i]);
      s.xb_key[i] = (int16_t)key;
      const int old = s.xb_state[i];
      const float* c = cum_xb + key * 36 + old * 6;
      const float u = uniform_of(sub, X, i, A.u_xb, inj_off);
      int ns = 0;
#pragma unroll
      for (int k = 5; k >= 0; --k)
        if (u < __ldg(c + k)) ns = k;
      const bool ob = old >= 1 && old <= 3, nbd = ns >= 1 && ns <= 3;
      const bool binding = !ob && nbd, unbinding = ob && !nbd;
      const bool occupied = s.thin_bound[tgt] >= 0;
      const bool can_bind = binding && perm && !occupied;
      const int ob_site = s.xb_bound[i];
      const int t1 = thin * T.n_sites + (ob_site < 0 ? 0 : (ob_site > T.n_sites - 1 ? T.n_sites - 1 : ob_site));
      atomicMax(&win1[t1], i);
      atomicMax(&s.win2[tgt], i);
      // stash the decision in fxb (as int bits): new state | can_bind<<4 | binding<<5 | unbinding<<6
      int code = ns | (can_bind << 4) | (binding << 5) | (unbinding << 6);
      reinterpret_cast<int*>(s.fxb)[i] = code;
    }
    __syncthreads();
    // STEP 1: the highest-index writer of each site decides whether it is cleared
    for (int i = tid; i < X; i += NT) {
      const int code = reinterpret_cast<int*>(s.fxb)[i];
      const int ob_site = s.xb_bound[i];
      const int thin = thin_of(i);
      const int t1 = thin * T.n_sites + (ob_site < 0 ? 0 : (ob_site > T.n_sites - 1 ? T.n_sites - 1 : ob_site));
      if (win1[t1] == i && (code & 64) && ob_site >= 0) s.thin_bound[t1] = -1;
    }
    __syncthreads();
    // STEP 2: the highest-index writer of each nearest site claims it if it binds
    for (int i = tid; i < X; i += NT) {
      const int code = reinterpret_cast<int*>(s.fxb)[i];
      const int thin = thin_of(i);
      const int near = s.xb_near[i];
      const int site = near < 0 ? 0 : (near > T.n_sites - 1 ? T.n_sites - 1 : near);
      const int tgt = thin * T.n_sites + site;
      if (s.win2[tgt] == i && (code & 16)) s.thin_bound[tgt] = (int16_t)i;
      int ns = code & 15;
      const bool can_bind = code & 16, binding = code & 32, unbinding = code & 64;
      if (can_bind) s.xb_bound[i] = (int16_t)near;
      else if (unbinding) s.xb_bound[i] = -1;
      if (binding && !can_bind) ns = 0;
      s.xb_state[i] = (int8_t)ns;
    }
    __syncthreads();
  }
};

}  // namespace mf
