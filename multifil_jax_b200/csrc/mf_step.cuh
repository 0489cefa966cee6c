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
  int drv_const;          // 1: z/pCa/ls hold one value for every step (zero: per-step traces)
  const float* params;    // [44]
  const float* z;         // [T], or [1] with drv_const
  const float* pCa;       // [T], or [1] with drv_const
  const float* ls;        // [T], or [1] with drv_const
  const uint32_t* key;    // [2] key at step 0
  float* metrics;         // [52*T]
  int* status;            // or NULL
  uint32_t* key_out;      // [2] or NULL
  float K_lat, nu, dt;
  // subpopulations (StepArgs::pop): K parameter rows, K fractions, per-head
  // and per-site population labels (NULL when unused)
  const float* pop_params;
  const float* pop_frac;
  const int8_t* xb_label;
  const int8_t* tm_label;
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
  PopShape pop;          // subpopulations of the batch (K <= 1: none)
};

constexpr int FLAG_DYN = 1, FLAG_PRECISE = 2, FLAG_ORIG_PRNG = 4;

// 4-byte asynchronous global -> shared copy (no register holds the value)
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
// Transposed warp reduction of 32 values per lane: after it lane l holds the
// warp total of value l (max for l < NMAX, sum otherwise).  Each of the five
// exchange steps halves the values a lane keeps, so it takes 31 shuffles
// where 32 separate butterfly reductions take 160.
template <int NMAX>
__device__ __forceinline__ float warp_reduce_transposed(float (&v)[32], int lane) {
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) {
    const bool up = (lane & o) != 0;
    const int base = lane & (32 - o);  // value index of position 0 after this step, minus j
#pragma unroll
    for (int j = 0; j < o; ++j) {
      const float send = up ? v[j] : v[j + o];
      const float keep = up ? v[j + o] : v[j];
      const float recv = __shfl_xor_sync(0xffffffffu, send, o);
      v[j] = base + j < NMAX ? fmax_nan(keep, recv) : keep + recv;
    }
  }
  return v[0];
}

__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax_nan(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Per-condition inputs of the table builder, kept in the CTA's shared memory
// (Smem::tab) so that a call passes one address and the per-call values.
struct TableCtx {
  const float* P;        // [44] wild-type parameter row
  const float* centers;  // [n_bins] bin centres
  int nb;                // n_bins
  float dtm;             // timestep (ms)
  int sq64;              // float64 squaring from this s on
  float* cum_tm;         // [kt*27*16]
  float* cum_xb;         // [kx*2*n_bins*36]
  float* pabs;           // [kx*2*n_bins*3]
  PopShape pop;
  const float* Pk;       // [K*44] population rows
  const float* fk;       // [K] fractions
};

// Shared-memory carve of one condition.
struct Smem {
  float* x;       // [N] node positions (precise mode: displacements)
  float* r;       // [N] residual / CG residual
  float* dx;      // [N] CG solution
  float* pv;      // [N] CG direction
  float* zz;      // [N] preconditioned residual / J p
  float* wv;      // [N] A u (precise-mode CG)
  float* sv;      // [N] A p (precise-mode CG)
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
  float* pabs;    // [2*n_bins*3] absorbing-chain entries read by the metrics (kept
                  // in the workspace between launches)
  float* coef;    // Thomas scan coefficients (thick fwd, thick back, thin fwd, thin back, inv)
  float* scan;    // per-warp scan reversal buffer (float32 mode)
  float* P;       // [44]
  float* red;     // reduction scratch [64]
  double* redd;   // [64]
  float* tvec;    // [4*n_thick] titin partials
  float* fdd;     // [X] df/dd per head (dynamic spacing)
  float* frdd;    // [X] d(radial)/dd per head (dynamic spacing)
  int16_t* blist; // [X] heads carrying force this step, increasing index
  int* hsite;     // [X] global site of a force-carrying head, else -1 (int32: the JVP reads
                  // three per node with a nine-word lane stride, free of bank conflicts)
  int16_t* site_h;// [2S] first two force-carrying heads of every site (over site)

  double* face_pos; // [n_thin*3*width] staged candidate positions, NaN = invalid (over site, win2)
  int8_t* face_mono;// [n_thin*3] 0 scan, 1 increasing, 2 decreasing, 3 no candidate
  int8_t* face_kl;  // [n_thin*3] first valid candidate
  int8_t* face_kh;  // [n_thin*3] last valid candidate
  int* nbound;    // [1] length of blist
  int* wsum;      // [32] per-warp counts of the compaction scan
  // pre-step (old_state) snapshot read by the metrics epilogue: shared memory
  // when the lattice leaves room, else the resident workspace arrays
  float* old_thick;  // [n_thick*n_crowns]
  int8_t* old_xbs;   // [X]
  int16_t* old_key;  // [X] table row (permissiveness, bin) of the pre-step geometry
  int16_t* xb_key;   // [X] table row used by the latest crossbridge sampling
  // subpopulations: K parameter rows and fractions, per-head / per-site
  // population labels (only when the batch has populations)
  float* Pk;         // [K*44]
  float* fk;         // [K]
  int8_t* xlab;      // [X] when the crossbridge tables are per population
  int8_t* tlab;      // [S] when the tropomyosin tables are per population
  TableCtx tab;      // the table builder's per-condition inputs
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

// Transition tables of one condition at (pCa, d), built by the whole CTA:
// the 27 tropomyosin row sums (shared) and, per crossbridge bin and
// permissiveness, the cumulative rows of expm(Q dt) ("sampling", global) or
// the three absorbing-chain entries the metrics read ("absorbing", global).
// Each matrix is one lane pair's work (expm_pair): lane h builds, keeps and
// stores rows h*N/2 ... of it.  Out of line: it runs only when pCa or the
// spacing changes, and its Pade arithmetic would otherwise sit in the step
// loop's code.  tm: the 27 tropomyosin tables; sampling / absorbing: the
// crossbridge tables of every key, or with `keys` only the nkeys listed ones
// (of the one kind selected), or with `keys` and both kinds selected every
// sampling key followed by the listed absorbing keys.  Work goes to the
// pairs in rounds of nt/2 matrices; every-key sampling work runs in
// descending bin order (table_key_of_order): the far bins, whose stiff
// generators take the most squarings, share the first round and the cheap
// central bins the last one.
//
// Subpopulations (pop, with the K population rows Pk and fractions fk):
// a blended family uses sum_k f_k Q_k, products and sums rounded one by one
// in population order from 0 (the reference's Python sum,
// transitions.py:580-585, 967-971); an explicit family keeps one table set
// per population, population-major (table key = population * (2 n_bins) +
// permissiveness * n_bins + bin; tropomyosin row = population * 27 + cfg).
// Population rows differ from P only in xb_* / tm_* rate fields.
template <int R, int C>
static __device__ __forceinline__ void blend_acc(float (&acc)[R][C], const float (&q)[R][C], float f) {
#pragma unroll
  for (int i = 0; i < R; ++i)
#pragma unroll
    for (int j = 0; j < C; ++j) acc[i][j] = __fadd_rn(acc[i][j], __fmul_rn(f, q[i][j]));
}

// The crossbridge table key (population * 2 n_bins + permissiveness * n_bins
// + bin) at position ord of the bin-major order ord = (bin * kx + population)
// * 2 + permissiveness.
__device__ __forceinline__ int table_key_of_order(int ord, int kx, int nb) {
  const int perm = ord & 1, q = ord >> 1, pk = q % kx, bin = q / kx;
  return pk * 2 * nb + perm * nb + bin;
}

static __device__ __noinline__ void build_tables_block(const TableCtx& c, float pCa, float d, bool tm, bool sampling,
                                                bool absorbing, const int16_t* keys, int nkeys, int tid, int nt) {
  const float* P = c.P;
  const float* centers = c.centers;
  const int nb = c.nb, sq64 = c.sq64;
  const float dtm = c.dtm;
  float* cum_tm = c.cum_tm;
  float* cum_xb = c.cum_xb;
  float* pabs = c.pabs;
  const PopShape pop = c.pop;
  const float* Pk = c.Pk;
  const float* fk = c.fk;
  const int h = tid & 1;                                  // which half of the rows
  const int pair = tid >> 1, npairs = nt >> 1;
  const unsigned pmask = 3u << (tid & 30);
  if (tm) {
    const int kt = pop.kt();
    const bool blend = pop.blend_tm();
    for (int m = pair; m < kt * 27; m += npairs) {
      const int cfg = m % 27, pk = m / 27;
      float q[2][4];
      if (blend) {
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) q[i][j] = 0.f;
        for (int k = 0; k < pop.K; ++k) {
          float qk[2][4];
          tm_generator_rows(Pk + k * kNParams, pCa, cfg, h, qk);
          blend_acc(q, qk, fk[k]);
        }
      } else {
        tm_generator_rows(kt > 1 ? Pk + pk * kNParams : P, pCa, cfg, h, q);
      }
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) q[i][j] = q[i][j] * dtm;
      expm_pair<4>(pmask, h, q, sq64);
#pragma unroll
      for (int i = 0; i < 2; ++i) cum4(q[i], cum_tm + m * 16 + 4 * (2 * h + i));
    }
  }
  const int kx = pop.kx(), nset = 2 * nb;  // keys of one population's set
  const int nall = kx * nset;
  const bool blend = pop.blend_xb();
  const bool all_then_list = keys && sampling && absorbing;
  const int nwork = keys ? nkeys + (all_then_list ? nall : 0) : (sampling ? nall : 0) + (absorbing ? nall : 0);
  for (int w = pair; w < nwork; w += npairs) {
    bool is_abs;
    int key;
    if (all_then_list) {
      is_abs = w >= nall;
      key = is_abs ? (int)keys[w - nall] : table_key_of_order(nall - 1 - w, kx, nb);
    } else if (keys) {
      is_abs = absorbing;
      key = keys[w];
    } else {
      is_abs = !sampling || w >= nall;
      key = is_abs && sampling ? w - nall : w;
    }
    const int pk = key / nset, k2 = key - pk * nset;
    const int bin = k2 % nb;
    const float perm = k2 >= nb ? 1.0f : 0.0f;
    float q[3][6];
    if (blend) {
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 6; ++j) q[i][j] = 0.f;
      for (int k = 0; k < pop.K; ++k) {
        float qk[3][6];
        xb_generator_rows(Pk + k * kNParams, pCa, centers[bin], d, perm, h, qk);
        blend_acc(q, qk, fk[k]);
      }
    } else {
      xb_generator_rows(kx > 1 ? Pk + pk * kNParams : P, pCa, centers[bin], d, perm, h, q);
    }
    if (is_abs) {  // the absorbing chain: rows 0 and 4 zeroed
#pragma unroll
      for (int j = 0; j < 6; ++j) q[h == 0 ? 0 : 1][j] = 0.f;
    }
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 6; ++j) q[i][j] = q[i][j] * dtm;
    expm_pair<6>(pmask, h, q, sq64);
    if (is_abs) {
      if (h == 1) {
        pabs[key * 3 + 0] = q[0][4];  // P_abs[3,4]
        pabs[key * 3 + 2] = q[0][0];  // P_abs[3,0]
      } else {
        pabs[key * 3 + 1] = q[2][0];  // P_abs[2,0]
      }
    } else {
#pragma unroll
      for (int i = 0; i < 3; ++i) cum6(q[i], cum_xb + key * 36 + 6 * (3 * h + i));
    }
  }
}

// The dynamic-spacing flag: a runtime member in kernels built for dynamic
// spacing (the initial equilibrium still holds the spacing fixed), a
// compile-time false elsewhere.
template <bool DY>
struct SimDyn {
  bool dyn;
  __device__ void set_dyn(bool v) { dyn = v; }
};
template <>
struct SimDyn<false> {
  static constexpr bool dyn = false;
  __device__ void set_dyn(bool) {}
};

template <int NT, bool PR, bool DY>
struct Sim : SimDyn<DY> {
  using SimDyn<DY>::dyn;
  static constexpr int NW = NT / 32;
  // Filaments longer than 128 nodes (8 per lane in the scans and CG passes)
  // run only in CTAs of 512 or more threads, which the host picks for them;
  // the smaller instances carry no code for them.
  static constexpr bool kWide = NT >= kWideThreads;
  // The lattice, the shared-memory carve and the layouts live in CTA-shared
  // structs at fixed addresses: reading a field is one shared load, and none
  // of the ~50 pointers and sizes occupies a register across the step loop.
  const TopoDev& T;
  const StepArgs& A;
  Smem& s;
  CoefLayout& cl;
  SlotLayout& L;
  char* ws;
  int b;        // caller row
  int tid, lane, warp;
  static constexpr bool precise = PR;
  bool part;
  bool regcg;   // register-resident precise Newton-CG (solve_regs)
  bool lazy_tab;  // dynamic spacing: build only the crossbridge table rows the heads read
  float Kl, nu_c, dtm;
  double zref;  // precise mode thin reference z
  float dvar;   // lattice spacing unknown (dynamic) / fixed spacing
  float d_ref;
  int status;
  int Tstride;
  int redbuf = 0;
#ifdef MF_PHASE_TIMING
  // diagnostic build only: thread 0's clock64() totals of solver sub-phases
  long long sub_t0 = 0;
  double* sub_acc = nullptr;  // the phase totals' shared array, slots 12..19
#define MF_SUB(k)                                               \
  do {                                                          \
    __syncthreads();                                            \
    if (tid == 0) {                                             \
      const long long now_ = clock64();                         \
      if ((k) >= 0) sub_acc[(k) < 0 ? 0 : (k)] += (double)(now_ - sub_t0); \
      sub_t0 = now_;                                            \
    }                                                           \
  } while (0)
#define MF_COUNT(k) (sub_acc[k] += 1.0)
#else
#define MF_SUB(k) do { } while (0)
#define MF_COUNT(k) do { } while (0)
#endif

  __device__ Sim(const TopoDev& t, const StepArgs& a, Smem& sm, CoefLayout& c, SlotLayout& l)
      : T(t), A(a), s(sm), cl(c), L(l) {}

  // ------------------------------------------------------------------
  // reductions
  // ------------------------------------------------------------------
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
  // The reference's lax.associative_scan dataflow (JAX's odd/even
  // recursion) for the b-components of an affine-map scan whose a-components
  // per tree node are precomputed (Acoef, ScanPlan level offsets), evaluated
  // in registers for one filament of n <= 32 E nodes (E = 4 or 8).  Lane L
  // holds level-l elements [L E/2^l, (L+1) E/2^l) for every level l below
  // log2(E) + 1 (w[l][]), and element L of every level above.  Up-sweep:
  // level l+1 element k = fmaf(A_l[2k+1], E_l[2k], E_l[2k+1]).  Down-sweep,
  // from the scanned level l+1 S: E_l[2k+1] = S[k],
  // E_l[2k] = fmaf(A_l[2k], S[k-1], E_l[2k]) for k >= 1.  The in-lane levels
  // need no data movement; the higher ones move by warp shuffles.
  template <int E>
  __device__ __forceinline__ void scan_regs(const ScanPlan& pl, const float* __restrict__ Acoef,
                                            float (&e)[E]) const {
    constexpr int LE = E == 8 ? 3 : 2;  // levels held inside a lane, above level 0
    constexpr int ML = LE + 6;          // levels of a 32 E-element scan
    static_assert(E == 4 || E == 8, "4 or 8 nodes per lane");
    int len[ML], off[ML];
    const int levels = pl.levels;
#pragma unroll
    for (int l = 0; l < ML; ++l) {
      len[l] = l < levels ? pl.len[l] : 0;
      off[l] = l < levels ? pl.off[l] : 0;
    }
    const int L = lane;
    float w[LE + 1][E];
#pragma unroll
    for (int i = 0; i < E; ++i) w[0][i] = e[i];
#pragma unroll
    for (int l = 0; l < LE; ++l) {
      const int C = E >> (l + 1);
#pragma unroll
      for (int j = 0; j < E / 2; ++j)
        if (j < C) {
          const int k = L * C + j;
          w[l + 1][j] = k < len[l + 1] ? fmaf(Acoef[off[l] + 2 * k + 1], w[l][2 * j], w[l][2 * j + 1]) : 0.f;
        }
    }
    float v[ML];
#pragma unroll
    for (int l = 0; l < ML; ++l) v[l] = 0.f;
    v[LE] = w[LE][0];
#pragma unroll
    for (int l = LE; l + 1 < ML; ++l) {
      const float a = __shfl_sync(0xffffffffu, v[l], (2 * L) & 31);
      const float b = __shfl_sync(0xffffffffu, v[l], (2 * L + 1) & 31);
      if (L < len[l + 1]) v[l + 1] = fmaf(Acoef[off[l] + 2 * L + 1], a, b);
    }
    // down-sweep from the top: level l from the scanned level l + 1
#pragma unroll
    for (int l = ML - 2; l >= LE; --l) {
      const int src = (L & 1) ? (L - 1) >> 1 : (L >> 1) - 1;
      const float sv = __shfl_sync(0xffffffffu, v[l + 1], src & 31);
      if (l + 1 < levels && L < len[l]) {
        if (L & 1) v[l] = sv;                                              // E[2k+1] = S[k]
        else if (L >= 2) v[l] = fmaf(Acoef[off[l] + L], sv, v[l]);         // E[2k] += A[2k] S[k-1]
      }
    }
    w[LE][0] = v[LE];
    // in-lane levels: S[k-1] of the lane's first k is the previous lane's last
#pragma unroll
    for (int l = LE - 1; l >= 0; --l) {
      const int C = E >> (l + 1);  // level l+1 elements per lane
      float last = w[l + 1][0];
#pragma unroll
      for (int j = 1; j < E / 2; ++j)
        if (j < C) last = w[l + 1][j];
      const float sp = __shfl_up_sync(0xffffffffu, last, 1);
      if (l + 1 < levels) {
#pragma unroll
        for (int j = 0; j < E / 2; ++j)
          if (j < C) {
            const int k = L * C + j;
            const float prev = j == 0 ? sp : w[l + 1][j > 0 ? j - 1 : 0];
            if (2 * k < len[l] && k >= 1) w[l][2 * j] = fmaf(Acoef[off[l] + 2 * k], prev, w[l][2 * j]);
            if (2 * k + 1 < len[l]) w[l][2 * j + 1] = w[l + 1][j];
          }
      }
    }
#pragma unroll
    for (int i = 0; i < E; ++i) e[i] = w[0][i];
  }

  // The same dataflow for 4 nodes per lane, written out level by level (the
  // form of the 128-node instances, which keeps fewer values live than the
  // general template).
  __device__ __forceinline__ void scan_regs4(const ScanPlan& pl, const float* __restrict__ Acoef,
                                            float (&e)[4]) const {
    constexpr int ML = 8;  // levels of a 128-element scan
    int len[ML], off[ML];
    const int levels = pl.levels;
#pragma unroll
    for (int l = 0; l < ML; ++l) {
      len[l] = l < levels ? pl.len[l] : 0;
      off[l] = l < levels ? pl.off[l] : 0;
    }
    const int L = lane;
    float l1[2];
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const int k = 2 * L + c;
      l1[c] = k < len[1] ? fmaf(Acoef[off[0] + 2 * k + 1], e[2 * c], e[2 * c + 1]) : 0.f;
    }
    float v[ML];
#pragma unroll
    for (int l = 0; l < ML; ++l) v[l] = 0.f;
    v[2] = L < len[2] ? fmaf(Acoef[off[1] + 2 * L + 1], l1[0], l1[1]) : 0.f;
#pragma unroll
    for (int l = 2; l + 1 < ML; ++l) {
      const float a = __shfl_sync(0xffffffffu, v[l], (2 * L) & 31);
      const float b = __shfl_sync(0xffffffffu, v[l], (2 * L + 1) & 31);
      if (L < len[l + 1]) v[l + 1] = fmaf(Acoef[off[l] + 2 * L + 1], a, b);
    }
    // down-sweep from the top: level l from the scanned level l + 1
#pragma unroll
    for (int l = ML - 2; l >= 2; --l) {
      const int src = (L & 1) ? (L - 1) >> 1 : (L >> 1) - 1;
      const float sv = __shfl_sync(0xffffffffu, v[l + 1], src & 31);
      if (l + 1 < levels && L < len[l]) {
        if (L & 1) v[l] = sv;                                              // E[2k+1] = S[k]
        else if (L >= 2) v[l] = fmaf(Acoef[off[l] + L], sv, v[l]);         // E[2k] += A[2k] S[k-1]
      }
    }
    {
      const float sp = __shfl_up_sync(0xffffffffu, v[2], 1);
      if (2 < levels) {
        if (2 * L + 1 < len[1]) l1[1] = v[2];
        if (2 * L < len[1] && L >= 1) l1[0] = fmaf(Acoef[off[1] + 2 * L], sp, l1[0]);
      }
    }
    {
      const float sp = __shfl_up_sync(0xffffffffu, l1[1], 1);
      if (1 < levels) {
        const int n0 = len[0];
        if (4 * L < n0 && L >= 1) e[0] = fmaf(Acoef[off[0] + 4 * L], sp, e[0]);
        if (4 * L + 1 < n0) e[1] = l1[0];
        if (4 * L + 2 < n0) e[2] = fmaf(Acoef[off[0] + 4 * L + 2], l1[0], e[2]);
        if (4 * L + 3 < n0) e[3] = l1[1];
      }
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
  __device__ __forceinline__ void thomas_regs(float (&y)[E], int n, const float* __restrict__ Af,
                                              const float* __restrict__ Ab, const float* __restrict__ inv) const {
    float a[E];
    const int i0 = lane * E;
    // forward: y[i] = a_f[i] * y[i-1] + r[i], y[-1] = 0
    float A = 1.f, Bv = 0.f;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int i = i0 + e;
      a[e] = i < n ? Af[i] : 1.f;
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
      y[e] = xp;
    }
  }
  template <int E>
  __device__ __forceinline__ void thomas_shfl(const float* in, float* out, int n, const float* Af,
                                              const float* Ab, const float* inv) {
    float y[E];
    const int i0 = lane * E;
#pragma unroll
    for (int e = 0; e < E; ++e) y[e] = i0 + e < n ? in[i0 + e] : 0.f;
    thomas_regs<E>(y, n, Af, Ab, inv);
#pragma unroll
    for (int e = 0; e < E; ++e)
      if (i0 + e < n) out[i0 + e] = y[e];
  }

  // out = M^{-1} in on this warp's own filaments (no block barrier needed).
  __device__ __forceinline__ void precondition_own(const float* in, float* out) {
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
        else if (!kWide || n <= 128) thomas_shfl<4>(in + base, out + base, n, Af, Ab, inv);
        else if constexpr (kWide) thomas_shfl<8>(in + base, out + base, n, Af, Ab, inv);
      }
      __syncwarp();
      return;
    }
    float* buf = s.scan + warp * (kWide ? scan_cap(T) : 128);  // this warp's reversal buffer
    __syncwarp();
    for (int f = warp; f < nf; f += NW) {
      const bool thick = f < T.n_thick;
      const int n = thick ? T.n_crowns : T.n_sites;
      const int base = thick ? f * T.n_crowns : T.n_thick_nodes + (f - T.n_thick) * T.n_sites;
      const ScanPlan& pl = thick ? T.plan_thick : T.plan_thin;
      const float* Af = s.coef + (thick ? cl.thick_fwd : cl.thin_fwd);
      const float* Ab = s.coef + (thick ? cl.thick_back : cl.thin_back);
      const float* inv = s.coef + (thick ? cl.thick_inv : cl.thin_inv);
      if (!kWide || n <= 128) thomas_tree<4>(in, out, base, n, pl, Af, Ab, inv, buf);
      else if constexpr (kWide) thomas_tree<8>(in, out, base, n, pl, Af, Ab, inv, buf);
    }
    __syncwarp();
  }

  // float32 Thomas solve of one filament in the reference's tree order:
  // forward scan in registers, (y * inv) reversed through this warp's
  // scratch, backward scan, reversed store.
  template <int E>
  __device__ __forceinline__ void thomas_tree(const float* in, float* out, int base, int n, const ScanPlan& pl,
                                              const float* Af, const float* Ab, const float* inv, float* buf) {
    float e[E];
#pragma unroll
    for (int c = 0; c < E; ++c) {
      const int i = E * lane + c;
      e[c] = i < n ? in[base + i] : 0.f;
    }
    if constexpr (E == 4) scan_regs4(pl, Af, e);
    else scan_regs<E>(pl, Af, e);
#pragma unroll
    for (int c = 0; c < E; ++c) {
      const int i = E * lane + c;
      if (i < n) buf[n - 1 - i] = e[c] * inv[i];
    }
    __syncwarp();
#pragma unroll
    for (int c = 0; c < E; ++c) {
      const int i = E * lane + c;
      e[c] = i < n ? buf[i] : 0.f;
    }
    __syncwarp();
    if constexpr (E == 4) scan_regs4(pl, Ab, e);
    else scan_regs<E>(pl, Ab, e);
#pragma unroll
    for (int c = 0; c < E; ++c) {
      const int i = E * lane + c;
      if (i < n) out[base + n - 1 - i] = e[c];
    }
  }

  // One-barrier block reduction of K floats (sum) with an optional max in
  // slot 0; double-buffered so consecutive reductions need no extra barrier.
  template <int K>
  __device__ __forceinline__ void reduce(float (&v)[K], bool max0) {
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = (max0 && k == 0) ? warp_max(v[k]) : warp_sum(v[k]);
    float* rb = s.red + kRedPartials * NW + redbuf * 96;  // clear of the metrics partials and the force slot
    redbuf ^= 1;
    if (lane == 0)
#pragma unroll
      for (int k = 0; k < K; ++k) rb[k * NW + warp] = v[k];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; ++k) {
      float t = rb[k * NW];
      for (int w = 1; w < NW; ++w) t = (max0 && k == 0) ? fmax_nan(t, rb[k * NW + w]) : t + rb[k * NW + w];
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
    const int gs = s.hsite[xb];
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
    arg = fmin_nan(fmax_nan(arg, -100.f), 100.f);
    const float Ft = fmax_nan(s.P[TITIN_A] * expf(arg), 0.f);
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
  // site), in increasing head index (block prefix scan, deterministic); the
  // global site of every such head (hsite, -1 for the others); per site the
  // number of such heads (win2) and the first two of them (site_h).  Node
  // owners gather the crossbridge terms of their sites from these lists:
  // sums of one or two heads are order-free, sites holding 3+ heads are
  // summed in head order (the reference adds in index order,
  // transitions/forces.py segment_sum).  Clears the per-head accumulator.
  __device__ __forceinline__ void build_bound_list() {
    const int X = T.total_xbs, S = T.n_sites_total, nsi = T.n_sites;
    int* __restrict__ cnt = s.win2;
    int16_t* __restrict__ site_h = s.site_h;
    // every caller ends its previous phase with a barrier (thick_step's
    // last scatter, the nearest-site search of the initial equilibrium)
    for (int g = tid; g < S; g += NT) cnt[g] = 0;
    __syncthreads();
    // each thread takes a run of consecutive heads, so one block-wide scan of
    // the per-thread counts places every head in increasing index order
    const int per = (X + NT - 1) / NT, i0 = tid * per;
    const int i1 = i0 + per < X ? i0 + per : X;
    int nf = 0;
    for (int i = i0; i < i1; ++i) {
      s.fxb[i] = 0.f;
      const int st = s.xb_state[i];
      const int bnd = s.xb_bound[i];
      const bool f = st >= 1 && st <= 3 && bnd >= 0;
      int gs = -1;
      if (f) {
        gs = thin_of(i) * nsi + bnd;
        const int k = atomicAdd(&cnt[gs], 1);
        if (k < 2) site_h[2 * gs + k] = (int16_t)i;
        else if (k == 2) status |= MF_MULTIBIND_BIT;
        ++nf;
      }
      s.hsite[i] = gs;
    }
    int incl = nf;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    if (lane == 31) s.wsum[warp] = incl;
    __syncthreads();
    int off = incl - nf, tot = 0;
    for (int w = 0; w < NW; ++w) {
      const int v = s.wsum[w];
      off += w < warp ? v : 0;
      tot += v;
    }
    for (int i = i0; i < i1; ++i)
      if (s.hsite[i] >= 0) s.blist[off++] = (int16_t)i;
    if (tid == 0) *s.nbound = tot;
    // the two heads of a site in head order (their slots came from the
    // atomic counter; a contracted multiply-add of the second term is not
    // symmetric, so the sums over them need one fixed order)
    uint32_t* pairs = reinterpret_cast<uint32_t*>(site_h);
    for (int g = tid; g < S; g += NT) {
      if (cnt[g] == 2) {
        const uint32_t w = pairs[g];
        if ((w >> 16) < (w & 0xffffu)) pairs[g] = (w >> 16) | (w << 16);
      }
    }
    __syncthreads();
  }

  // -sum of val(h) over the force-carrying heads of site g: in head order
  // for 3+ heads (blist is sorted), order-free otherwise; starts from 0 like
  // the reference's segment_sum.
  template <class Val>
  __device__ __forceinline__ float site_sum(int g, Val&& val) const {
    const int c = s.win2[g];
    float acc = 0.f;
    if (c < 3) {
      // site_h[2g], site_h[2g+1] in one word, in head order (build_bound_list)
      const uint32_t pair = reinterpret_cast<const uint32_t*>(s.site_h)[g];
      const int h0 = (int)(pair & 0xffffu), h1 = (int)(pair >> 16);
      if (c >= 1) acc = acc + (-val(h0));
      if (c >= 2) acc = acc + (-val(h1));
      return acc;
    }
    const int nb = *s.nbound;
    for (int k = 0; k < nb; ++k) {
      const int h = s.blist[k];
      if (s.hsite[h] == g) acc = acc + (-val(h));
    }
    return acc;
  }

  // Residual F(x) into s.r (own nodes); caches df/dx per bound head and the
  // titin partials for the JVPs of the next Newton iteration.  Returns max|F|
  // over the augmented vector; *frad = radial residual, *jdd = dF_rad/dd.
  // In precise mode the node forces are accumulated in float64.
  __device__ __forceinline__ float residual(float zl, float d, float* frad, float* jdd, int bad_in, int* bad_out) {
    const int nb = *s.nbound;
    const int nthk = T.n_thick, ncr = T.n_crowns, nsi = T.n_sites, ntn = T.n_thick_nodes, nxb = T.nxb;
    const float* __restrict__ x = s.x;
    float* __restrict__ r = s.r;
    float* __restrict__ fxb = s.fxb;
    float* __restrict__ tvec = s.tvec;
    float rad_part = 0.f, jdd_part = 0.f;
    const int any_bad = __syncthreads_or(bad_in);
    if (bad_out) *bad_out = any_bad;
    for (int k = tid; k < nb; k += NT) {
      const int i = s.blist[k];
      float f, fx, fd, frd, fr;
      xb_force(i, d, f, fx, fd, frd, fr);
      fxb[i] = f;
      s.fdx[i] = fx;
      if (dyn) {
        s.fdd[i] = fd;
        s.frdd[i] = frd;
        rad_part += fr;
        jdd_part += frd;
      }
    }
    // titin on the last threads: the bound heads above fill the first ones
    if (NT - 1 - tid < nthk) {
      const int th = NT - 1 - tid;
      float ax, a_x, a_d, r_d, rad;
      titin(th, zl, d, ax, a_x, a_d, r_d, rad);
      tvec[th] = ax;
      tvec[nthk + th] = a_x;
      tvec[2 * nthk + th] = a_d;
      tvec[3 * nthk + th] = r_d;
      if (dyn) {
        rad_part += rad;
        jdd_part += r_d;
      }
    }
    __syncthreads();
    const float kth = s.P[THICK_K], ktn = s.P[THIN_K];
    const float* __restrict__ crest = T.crown_rest;
    const float* __restrict__ brest = T.bind_rest;
    const float* __restrict__ thc = T.thick_c;
    const float* __restrict__ tnc = T.thin_c;
    const double zoff = (double)zl - zref;
    float fmax = 0.f;
    own_nodes([&](int i, int f, int j, bool thick) {
      double F;
      if (thick) {
        float xsum = fxb[i * nxb];
        for (int q = 1; q < nxb; ++q) xsum += fxb[i * nxb + q];
        if (!precise) {
          const float xm = j > 0 ? x[i - 1] : 0.f;
          const float sp_c = ((x[i] - xm) - crest[i]) * kth;
          const float sp_n = (j + 1 < ncr) ? ((x[i + 1] - x[i]) - crest[i + 1]) * kth : tvec[f];
          F = (double)((sp_n - sp_c) + xsum);
        } else {
          const double um = j > 0 ? (double)x[i - 1] : 0.0;
          const double e_c = ((double)x[i] - um) + (double)thc[i];
          const double spn = (j + 1 < ncr) ? (((double)x[i + 1] - (double)x[i]) + (double)thc[i + 1]) * (double)kth
                                           : (double)tvec[f];
          F = (spn - e_c * (double)kth) + (double)xsum;
        }
      } else {
        const int g = i - ntn;
        const float acc = site_sum(g, [&](int h) { return fxb[h]; });
        if (!precise) {
          const float xn = (j + 1 < nsi) ? x[i + 1] : zl;
          const float sp_j = ((xn - x[i]) - brest[g]) * ktn;
          const float sp_m = j > 0 ? ((x[i] - x[i - 1]) - brest[g - 1]) * ktn : 0.f;
          F = (double)((sp_j - sp_m) + acc);
        } else {
          const double un = (j + 1 < nsi) ? (double)x[i + 1] : 0.0;
          double e_j = (un - (double)x[i]) + (double)tnc[g];
          if (j + 1 == nsi) e_j += zoff;  // anchor vs reference z
          const double e_m = j > 0 ? ((double)x[i] - (double)x[i - 1]) + (double)tnc[g - 1] : 0.0;
          F = (e_j - e_m) * (double)ktn + (double)acc;
        }
      }
      r[i] = (float)F;
      fmax = fmax_nan(fmax, (float)fabs(F));
    });
    float v[3] = {fmax, rad_part, jdd_part};
    reduce<3>(v, true);
    float m = v[0];
    if (dyn) {
      const float Fr = -Kl * (d - d_ref) + (-v[1]);
      *frad = Fr;
      m = fmax_nan(m, fabsf(Fr));
      if (jdd) *jdd = -Kl - v[2];
    }
    return m;
  }

  // out = -(J [v, vd]) on own nodes; returns the augmented dot(v, out) and
  // *out_d the radial component.  The crossbridge couplings are gathered by
  // the node owners (each crown from its own heads, each site from the heads
  // bound to it), so one barrier before and the reduction after are all the
  // synchronisation.  The same reduction returns the block sum of
  // extra_part in *extra when extra is given.
  __device__ __forceinline__ float neg_jvp(const float* __restrict__ v, float vd, float* __restrict__ out, float* out_d,
                           float extra_part = 0.f, float* extra = nullptr) {
    const int nthk = T.n_thick, ncr = T.n_crowns, nsi = T.n_sites, ntn = T.n_thick_nodes, nxb = T.nxb;
    const float* __restrict__ fdx = s.fdx;
    const float* __restrict__ fdd = s.fdd;
    const float* __restrict__ frdd = s.frdd;
    const int* __restrict__ hsite = s.hsite;
    const float* __restrict__ tvec = s.tvec;
    const float kth = s.P[THICK_K], ktn = s.P[THIN_K];
    float rad_part = 0.f, dot = 0.f;
    auto head_w = [&](int h, float dxd) {
      float w = fdx[h] * dxd;
      if (dyn) w = w + fdd[h] * vd;
      return w;
    };
    __syncthreads();  // v complete
    own_nodes([&](int i, int f, int j, bool thick) {
      float J;
      const float vi = v[i];
      if (thick) {
        const float vm = j > 0 ? v[i - 1] : 0.f;
        const float sc = (vi - vm) * kth;
        float sn;
        if (j + 1 < ncr) sn = (v[i + 1] - vi) * kth;
        else {
          sn = tvec[nthk + f] * vi;
          if (dyn) {
            sn = sn + tvec[2 * nthk + f] * vd;
            rad_part += tvec[2 * nthk + f] * vi - tvec[3 * nthk + f] * vd;
          }
        }
        float xs = 0.f;
        for (int q = 0; q < nxb; ++q) {
          const int h = i * nxb + q;
          const int g = hsite[h];
          float w = 0.f;
          if (g >= 0) {
            const float dxd = v[ntn + g] - vi;
            w = head_w(h, dxd);
            if (dyn) rad_part += -(fdd[h] * dxd) - frdd[h] * vd;
          }
          xs = q == 0 ? w : xs + w;
        }
        J = (sn - sc) + xs;
      } else {
        const int g = i - ntn;
        const float vn = (j + 1 < nsi) ? v[i + 1] : 0.f;
        const float sj = (vn - vi) * ktn;
        const float sm = j > 0 ? (vi - v[i - 1]) * ktn : 0.f;
        J = (sj - sm) + site_sum(g, [&](int h) { return head_w(h, vi - v[h / nxb]); });
      }
      const float o = -J;
      out[i] = o;
      dot = fmaf(vi, o, dot);
    });
    float r3[3] = {dot, rad_part, extra_part};
    if (extra) {
      reduce<3>(r3, false);
      *extra = r3[2];
    } else {
      float r2[2] = {dot, rad_part};
      reduce<2>(r2, false);
      r3[0] = r2[0];
      r3[1] = r2[1];
    }
    if (dyn) {
      const float od = -(r3[1] + (-Kl) * vd);
      *out_d = od;
      return r3[0] + vd * od;
    }
    return r3[0];
  }

  // ------------------------------------------------------------------
  // Newton-CG (solver.py:329-427, 599-656).  Every piece (residual,
  // preconditioner, JVP) has one call site per solver, so each is inlined
  // once: the first Newton residual and the later ones share the loop top,
  // the initial preconditioned residual and the in-loop ones share the CG
  // loop body.
  // ------------------------------------------------------------------
  __device__ __forceinline__ void solve(float zl, float& d, double& resid, int& iters, bool dyn_jdd) {
    if constexpr (PR) {
      if (regcg) solve_regs(zl, d, resid, iters, dyn_jdd);
      else solve_cg_gear(zl, d, resid, iters, dyn_jdd);
    } else {
      solve_std(zl, d, resid, iters, dyn_jdd);
    }
  }

  // float32 mode: the reference's PCG recurrences and association orders.
  __device__ __forceinline__ void solve_std(float zl, float& d, double& resid, int& iters, bool dyn_jdd) {
    const float tol = fmax_nan(s.P[SOLVER_TOL], fmax_nan(s.P[THICK_K] * 1e-4f, 0.25f));
    const int n_cg = A.n_cg, n_newton = A.n_newton;
    float* __restrict__ xv = s.x;
    float* __restrict__ rv = s.r;
    float* __restrict__ zv = s.zz;
    float* __restrict__ pv = s.pv;
    float* __restrict__ dxv = s.dx;
    float frad = 0.f, jdd = 0.f, J_dd_inv = 0.f, fmx = 0.f;
    int it = 0, bad = 0, bad_local = 0;
    for (int nw = 0;; ++nw) {
      MF_SUB(-1);
      fmx = residual(zl, d, &frad, nw == 0 ? &jdd : nullptr, bad_local, nw == 0 ? nullptr : &bad);
      MF_SUB(0);
      if (nw == 0) {
        // exact radial diagonal at the pre-solve point (solver.py:633-638)
        J_dd_inv = dyn_jdd ? -1.0f / jdd : 0.f;
      } else if (bad) {
        status |= MF_NONFINITE_BIT;
      }
      it = nw;
      if (!(fmx > tol && nw < n_newton)) break;
      if (tid == 0) MF_COUNT(4);
      float r_d = frad, z_d = 0.f, p_d = 0.f, dx_d = 0.f, Ap_d = 0.f, rz = 0.f;
      for (int k = -1; k < n_cg; ++k) {
        if (k >= 0) {
          MF_SUB(-1);
          const float pAp = neg_jvp(pv, p_d, zv, &Ap_d);
          MF_SUB(2);
          if (tid == 0) MF_COUNT(3);
          const float alpha = rz / (pAp + 1e-30f);
          own_nodes([&](int i, int, int, bool) {
            dxv[i] = fmaf(alpha, pv[i], dxv[i]);
            rv[i] = rv[i] - alpha * zv[i];
          });
          dx_d = fmaf(alpha, p_d, dx_d);
          r_d = r_d - alpha * Ap_d;
          if (k + 1 == n_cg) break;  // the last direction update is never used
        }
        MF_SUB(-1);
        precondition_own(rv, zv);
        MF_SUB(1);
        float rzp[1] = {0.f};
        own_nodes([&](int i, int, int, bool) { rzp[0] = fmaf(rv[i], zv[i], rzp[0]); });
        if (dyn) z_d = J_dd_inv * r_d;
        reduce<1>(rzp, false);
        const float rz_new = rzp[0] + (dyn ? r_d * z_d : 0.f);
        if (k < 0) {
          own_nodes([&](int i, int, int, bool) {
            pv[i] = zv[i];
            dxv[i] = n_cg == 0 ? zv[i] : 0.f;
          });
          p_d = z_d;
          if (n_cg == 0) dx_d = z_d;
        } else {
          const float beta = rz_new / (rz + 1e-30f);
          own_nodes([&](int i, int, int, bool) { pv[i] = fmaf(beta, pv[i], zv[i]); });
          p_d = fmaf(beta, p_d, z_d);
        }
        rz = rz_new;
      }
      // x += dx with non-finite entries zeroed
      bad_local = 0;
      own_nodes([&](int i, int, int, bool) {
        float v = dxv[i];
        if (!isfinite(v)) { v = 0.f; bad_local = 1; }
        xv[i] = xv[i] + v;
      });
      if (dyn) {
        float v = dx_d;
        if (!isfinite(v)) v = 0.f;
        d = fmax_nan(d + v, 1.0f);
      }
    }
    resid = fmx;
    iters = it;
    if (!isfinite(fmx)) status |= MF_NONFINITE_BIT;
  }

  // Precise-mode CG step on one filament of this warp, lane-contiguous
  // layout (lane owns nodes [lane*E, lane*E+E)).  With update: the
  // Chronopoulos-Gear recurrences p = u + beta p, s = w + beta s,
  // dx += alpha p, r -= alpha s (first: p = u, s = w, dx = alpha u).  Then,
  // unless last, u = M^{-1} r by the register Thomas solve; returns this
  // lane's share of (r, u).  last: x += dx (non-finite entries zeroed).
  template <int E>
  __device__ __forceinline__ float cg_filament(int base, int n, const float* __restrict__ Af,
                                               const float* __restrict__ Ab, const float* __restrict__ inv,
                                               float alpha, float beta, bool update, bool first, bool last,
                                               int& bad) {
    float* __restrict__ r = s.r + base;
    float* __restrict__ u = s.zz + base;
    float* __restrict__ p = s.pv + base;
    float* __restrict__ sv = s.sv + base;
    float* __restrict__ dx = s.dx + base;
    const float* __restrict__ w = s.wv + base;
    float y[E], rr[E];
    const int i0 = lane * E;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int i = i0 + e;
      float ri = 0.f;
      if (i < n) {
        ri = r[i];
        if (update) {
          const float ui = u[i], wi = w[i];
          const float pi = first ? ui : fmaf(beta, p[i], ui);
          const float si = first ? wi : fmaf(beta, sv[i], wi);
          const float di = first ? alpha * pi : fmaf(alpha, pi, dx[i]);
          ri = ri - alpha * si;
          if (last) {
            float v = di;
            if (!isfinite(v)) { v = 0.f; bad = 1; }
            float* __restrict__ x = s.x + base;
            x[i] = x[i] + v;
          } else {
            p[i] = pi;
            sv[i] = si;
            dx[i] = di;
            r[i] = ri;
          }
        }
      }
      rr[e] = ri;
      y[e] = ri;
    }
    if (last) return 0.f;
    thomas_regs<E>(y, n, Af, Ab, inv);
    float g = 0.f;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int i = i0 + e;
      if (i < n) {
        u[i] = y[e];
        g = fmaf(rr[e], y[e], g);
      }
    }
    return g;
  }

  __device__ __forceinline__ float cg_pass(float alpha, float beta, bool update, bool first, bool last, int& bad) {
    const int nthk = T.n_thick, nf = T.n_thick + T.n_thin, ncr = T.n_crowns, nsi = T.n_sites;
    const int ntn = T.n_thick_nodes;
    float g = 0.f;
    __syncwarp();
    for (int f = warp; f < nf; f += NW) {
      const bool thick = f < nthk;
      const int n = thick ? ncr : nsi;
      const int base = thick ? f * ncr : ntn + (f - nthk) * nsi;
      const float* Af = s.coef + (thick ? cl.thick_fwd : cl.thin_fwd);
      const float* Ab = s.coef + (thick ? cl.thick_back : cl.thin_back);
      const float* inv = s.coef + (thick ? cl.thick_inv : cl.thin_inv);
      if (n <= 64) g += cg_filament<2>(base, n, Af, Ab, inv, alpha, beta, update, first, last, bad);
      else if (n <= 96) g += cg_filament<3>(base, n, Af, Ab, inv, alpha, beta, update, first, last, bad);
      else if (!kWide || n <= 128) g += cg_filament<4>(base, n, Af, Ab, inv, alpha, beta, update, first, last, bad);
      else if constexpr (kWide) g += cg_filament<8>(base, n, Af, Ab, inv, alpha, beta, update, first, last, bad);
    }
    __syncwarp();
    return g;
  }

  // Precise mode: the same truncated preconditioned CG in the
  // Chronopoulos-Gear arrangement (identical iterates in exact arithmetic):
  // w = A u is formed right after u, and (r, u), (w, u) are reduced
  // together, so an iteration costs the JVP barrier plus one reduction.
  // alpha_k = gamma_k / (delta_k - beta_k gamma_k / alpha_{k-1}) uses
  // (p_k, A p_k) = (u_k, A u_k) - beta_k^2 (p_{k-1}, A p_{k-1}).
  __device__ __forceinline__ void solve_cg_gear(float zl, float& d, double& resid, int& iters, bool dyn_jdd) {
    const float tol = fmax_nan(s.P[SOLVER_TOL], fmax_nan(s.P[THICK_K] * 1e-4f, 0.25f));
    const int n_cg = A.n_cg, n_newton = A.n_newton;
    float frad = 0.f, jdd = 0.f, J_dd_inv = 0.f, fmx = 0.f;
    int it = 0, bad = 0, bad_local = 0;
    for (int nw = 0;; ++nw) {
      MF_SUB(-1);
      fmx = residual(zl, d, &frad, nw == 0 ? &jdd : nullptr, bad_local, nw == 0 ? nullptr : &bad);
      MF_SUB(0);
      if (nw == 0) J_dd_inv = dyn_jdd ? -1.0f / jdd : 0.f;
      else if (bad) status |= MF_NONFINITE_BIT;
      it = nw;
      if (!(fmx > tol && nw < n_newton)) break;
      bad_local = 0;
      float r_d = frad, u_d = 0.f, w_d = 0.f, p_d = 0.f, s_d = 0.f, dx_d = 0.f;
      float alpha = 0.f, gamma = 0.f, gamma_old = 1.f, delta = 0.f;
      for (int k = -1; k < n_cg; ++k) {
        const bool first = k == 0, last = k + 1 == n_cg;
        float beta = 0.f;
        if (first) {
          alpha = gamma / (delta + 1e-30f);
        } else if (k > 0) {
          beta = gamma / (gamma_old + 1e-30f);
          alpha = gamma / (delta - beta * gamma / alpha + 1e-30f);
        }
        // k = -1: u = M^-1 r;  k >= 0: the recurrences, then u = M^-1 r
        MF_SUB(-1);
        const float gpart = cg_pass(alpha, beta, k >= 0, first, last && k >= 0, bad_local);
        MF_SUB(1);
        if (k >= 0) {
          p_d = first ? u_d : fmaf(beta, p_d, u_d);
          s_d = first ? w_d : fmaf(beta, s_d, w_d);
          dx_d = first ? alpha * p_d : fmaf(alpha, p_d, dx_d);
          r_d = r_d - alpha * s_d;
          if (last) break;
          gamma_old = gamma;
        }
        if (dyn) u_d = J_dd_inv * r_d;
        if (n_cg == 0) break;
        // w = A u, gamma = (r, u), delta = (u, w)
        MF_SUB(-1);
        delta = neg_jvp(s.zz, u_d, s.wv, &w_d, gpart, &gamma);
        MF_SUB(2);
        if (dyn) gamma += r_d * u_d;
      }
      if (n_cg == 0) {  // the preconditioned residual is the step
        float* __restrict__ xv = s.x;
        const float* __restrict__ uv = s.zz;
        __syncwarp();
        own_nodes([&](int i, int, int, bool) {
          float v = uv[i];
          if (!isfinite(v)) { v = 0.f; bad_local = 1; }
          xv[i] = xv[i] + v;
        });
        dx_d = u_d;
      }
      if (dyn) {
        float v = dx_d;
        if (!isfinite(v)) v = 0.f;
        d = fmax_nan(d + v, 1.0f);
      }
      if (tid == 0) MF_COUNT(4);
    }
    resid = fmx;
    iters = it;
    if (!isfinite(fmx)) status |= MF_NONFINITE_BIT;
  }
  static constexpr int MF_NONFINITE_BIT = 1, MF_MULTIBIND_BIT = 8;
  // ------------------------------------------------------------------
  // Register-resident precise Newton-CG (lattices with at most RF filaments
  // per warp and filaments of at most 32*RE nodes, crowns of 3 heads).
  // Lane l of a warp owns nodes [l*RE, l*RE+RE) of each of its filaments;
  // the CG vectors r, p, s, u, w, dx of those nodes stay in registers for
  // the whole solve, only u (read by the node's neighbours and partners)
  // and x (read by the head forces) are written to shared memory.  The
  // crossbridge coupling of every node is a fixed list of <= 3 partner
  // nodes built once per step (nb), so the JVP has no
  // dependent index chains.  Same Chronopoulos-Gear recurrences as
  // solve_cg_gear.
  // ------------------------------------------------------------------
  // RF filaments per warp (regcg_rf): one at 384 threads (a 2x2 lattice has
  // 12 filaments for 12 warps), three at 512 (3x3: 33, 4x4: 48), two otherwise
  static constexpr int RE = 3, RF = regcg_rf(NT);
  using RVec = float[RF][RE];

  __device__ __forceinline__ bool slot(int k, int& base, int& n, int& f, bool& thick) const {
    f = warp + k * NW;
    thick = f < T.n_thick;
    n = thick ? T.n_crowns : T.n_sites;
    base = thick ? f * T.n_crowns : T.n_thick_nodes + (f - T.n_thick) * T.n_sites;
    return f < T.n_thick + T.n_thin;
  }

  // F(x) of the lane's nodes into r (float64 accumulation, as residual());
  // returns max|F| over the augmented vector.
  __device__ __forceinline__ float residual_regs(float zl, float d, float* frad, float* jdd, int bad_in, int* bad_out, RVec& r) {
    const int nb = *s.nbound;
    const int nthk = T.n_thick;
    const float* __restrict__ x = s.x;
    float* __restrict__ fxb = s.fxb;
    float* __restrict__ tvec = s.tvec;
    float rad_part = 0.f, jdd_part = 0.f;
    const int any_bad = __syncthreads_or(bad_in);
    if (bad_out) *bad_out = any_bad;
    for (int k = tid; k < nb; k += NT) {
      const int i = s.blist[k];
      float f, fx, fd, frd, fr;
      xb_force(i, d, f, fx, fd, frd, fr);
      fxb[i] = f;
      s.fdx[i] = fx;
      if (dyn) {
        s.fdd[i] = fd;
        s.frdd[i] = frd;
        rad_part += fr;
        jdd_part += frd;
      }
    }
    // titin on the last threads: the bound heads above fill the first ones
    if (NT - 1 - tid < nthk) {
      const int th = NT - 1 - tid;
      float ax, a_x, a_d, r_d, rad;
      titin(th, zl, d, ax, a_x, a_d, r_d, rad);
      tvec[th] = ax;
      tvec[nthk + th] = a_x;
      tvec[2 * nthk + th] = a_d;
      tvec[3 * nthk + th] = r_d;
      if (dyn) {
        rad_part += rad;
        jdd_part += r_d;
      }
    }
    __syncthreads();
    const double kth = (double)s.P[THICK_K], ktn = (double)s.P[THIN_K];
    const float* __restrict__ thc = T.thick_c;
    const float* __restrict__ tnc = T.thin_c;
    const double zoff = (double)zl - zref;
    const int ntn = T.n_thick_nodes;
    constexpr int nxb = 3;
    float fmax = 0.f;
#pragma unroll
    for (int k = 0; k < RF; ++k) {
      int base, n, f;
      bool thick;
      const bool ok = slot(k, base, n, f, thick);
#pragma unroll
      for (int e = 0; e < RE; ++e) {
        const int j = lane * RE + e;
        float Fv = 0.f;
        if (ok && j < n) {
          const int i = base + j;
          const double xi = (double)x[i];
          const double xm = j > 0 ? (double)x[i - 1] : 0.0;
          const double xn = j + 1 < n ? (double)x[i + 1] : 0.0;
          double F;
          if (thick) {
            float xsum = fxb[i * nxb];
            for (int q = 1; q < nxb; ++q) xsum += fxb[i * nxb + q];
            const double e_c = (xi - xm) + (double)thc[i];
            const double spn = j + 1 < n ? ((xn - xi) + (double)thc[i + 1]) * kth : (double)tvec[f];
            F = (spn - e_c * kth) + (double)xsum;
          } else {
            const int g = i - ntn;
            float acc = 0.f;
            acc = site_sum(g, [&](int h) { return fxb[h]; });
            double e_j = (xn - xi) + (double)tnc[g];
            if (j + 1 == n) e_j += zoff;
            const double e_m = j > 0 ? (xi - xm) + (double)tnc[g - 1] : 0.0;
            F = (e_j - e_m) * ktn + (double)acc;
          }
          Fv = (float)F;
          fmax = fmax_nan(fmax, (float)fabs(F));
        }
        r[k][e] = Fv;
      }
    }
    float m;
    if constexpr (!DY) {
      float v[1] = {fmax};
      reduce<1>(v, true);
      return v[0];
    }
    float v[3] = {fmax, rad_part, jdd_part};
    reduce<3>(v, true);
    m = v[0];
    if (dyn) {
      const float Fr = -Kl * (d - d_ref) + (-v[1]);
      *frad = Fr;
      m = fmax_nan(m, fabsf(Fr));
      if (jdd) *jdd = -Kl - v[2];
    }
    return m;
  }

  // u = M^-1 r on the lane's nodes (register Thomas solves), u also stored
  // to shared memory; returns the lane's share of (r, u).
  __device__ __forceinline__ float precond_regs(const RVec& r, RVec& u) {
    float g = 0.f;
#pragma unroll
    for (int k = 0; k < RF; ++k) {
      int base, n, f;
      bool thick;
      if (!slot(k, base, n, f, thick)) break;
      const float* Af = s.coef + (thick ? cl.thick_fwd : cl.thin_fwd);
      const float* Ab = s.coef + (thick ? cl.thick_back : cl.thin_back);
      const float* inv = s.coef + (thick ? cl.thick_inv : cl.thin_inv);
      float y[RE];
#pragma unroll
      for (int e = 0; e < RE; ++e) y[e] = r[k][e];
      thomas_regs<RE>(y, n, Af, Ab, inv);
      float* __restrict__ us = s.zz + base;
#pragma unroll
      for (int e = 0; e < RE; ++e) {
        const int j = lane * RE + e;
        u[k][e] = j < n ? y[e] : 0.f;
        if (j < n) {
          us[j] = y[e];
          g = fmaf(r[k][e], y[e], g);
        }
      }
    }
    return g;
  }

  // w = -J [u, ud] on the lane's nodes; returns (u, w) (augmented) and the
  // block sum of extra_part in *extra, *w_d the radial component.
  __device__ __forceinline__ float jvp_regs(const RVec& u, float ud, RVec& w, float* w_d, float extra_part, float* extra) {
    const int nthk = T.n_thick;
    constexpr int nxb = 3;
    const float* __restrict__ us = s.zz;
    const float* __restrict__ fdx = s.fdx;
    const float* __restrict__ fdd = s.fdd;
    const float* __restrict__ frdd = s.frdd;
    const float* __restrict__ tvec = s.tvec;
    const int* __restrict__ hsite = s.hsite;
    const int ntn = T.n_thick_nodes;
    const float kth = s.P[THICK_K], ktn = s.P[THIN_K];
    float rad_part = 0.f, dot = 0.f;
    __syncthreads();  // u of every node stored
#pragma unroll
    for (int k = 0; k < RF; ++k) {
      int base, n, f;
      bool thick;
      const bool ok = slot(k, base, n, f, thick);
      const float left = __shfl_up_sync(0xffffffffu, u[k][RE - 1], 1);
      const float right = __shfl_down_sync(0xffffffffu, u[k][0], 1);
#pragma unroll
      for (int e = 0; e < RE; ++e) {
        const int j = lane * RE + e;
        float o = 0.f;
        if (ok && j < n) {
          const int i = base + j;
          const float vi = u[k][e];
          const float vm = j == 0 ? 0.f : (e > 0 ? u[k][e - 1] : left);
          const float vn = j + 1 >= n ? 0.f : (e + 1 < RE ? u[k][e + 1] : right);
          float J;
          if (thick) {
            const float sc = (vi - vm) * kth;
            float sn;
            if (j + 1 < n) sn = (vn - vi) * kth;
            else {
              sn = tvec[nthk + f] * vi;
              if (dyn) {
                sn = sn + tvec[2 * nthk + f] * ud;
                rad_part += tvec[2 * nthk + f] * vi - tvec[3 * nthk + f] * ud;
              }
            }
            float xs = 0.f;
#pragma unroll
            for (int q = 0; q < 3; ++q) {
              const int h = i * nxb + q;
              const int gq = hsite[h];
              float wq = 0.f;
              if (gq >= 0) {
                const int pn = ntn + gq;
                const float dxd = us[pn] - vi;
                wq = fdx[h] * dxd;
                if (dyn) {
                  wq = wq + fdd[h] * ud;
                  rad_part += -(fdd[h] * dxd) - frdd[h] * ud;
                }
              }
              xs = q == 0 ? wq : xs + wq;
            }
            J = (sn - sc) + xs;
          } else {
            const float sj = (vn - vi) * ktn;
            const float sm = j > 0 ? (vi - vm) * ktn : 0.f;
            auto head_w = [&](int h, float vc) {
              float wh = fdx[h] * (vi - vc);
              if (dyn) wh = wh + fdd[h] * ud;
              return wh;
            };
            const float acc = site_sum(i - ntn, [&](int h) { return head_w(h, us[h / nxb]); });
            J = (sj - sm) + acc;
          }
          o = -J;
          dot = fmaf(vi, o, dot);
        }
        w[k][e] = o;
      }
    }
    if constexpr (!DY) {
      float r2[2] = {dot, extra_part};
      reduce<2>(r2, false);
      *extra = r2[1];
      return r2[0];
    }
    float r3[3] = {dot, rad_part, extra_part};
    reduce<3>(r3, false);
    *extra = r3[2];
    if (dyn) {
      const float od = -(r3[1] + (-Kl) * ud);
      *w_d = od;
      return r3[0] + ud * od;
    }
    return r3[0];
  }

  __device__ __forceinline__ void solve_regs(float zl, float& d, double& resid, int& iters, bool dyn_jdd) {
    const float tol = fmax_nan(s.P[SOLVER_TOL], fmax_nan(s.P[THICK_K] * 1e-4f, 0.25f));
    RVec r;
    const int n_cg = A.n_cg, n_newton = A.n_newton;
    float frad = 0.f, jdd = 0.f, J_dd_inv = 0.f, fmx = 0.f;
    int it = 0, bad = 0, bad_local = 0;
    for (int nw = 0;; ++nw) {
      MF_SUB(-1);
      fmx = residual_regs(zl, d, &frad, nw == 0 ? &jdd : nullptr, bad_local, nw == 0 ? nullptr : &bad, r);
      MF_SUB(0);
      if (nw == 0) J_dd_inv = dyn_jdd ? -1.0f / jdd : 0.f;
      else if (bad) status |= MF_NONFINITE_BIT;
      it = nw;
      if (!(fmx > tol && nw < n_newton)) break;
      // The CG vectors live within one Newton iteration: the first update is
      // peeled off the loop so that none of them is live across the
      // residual evaluation.  n_cg >= 1 on this path.
      RVec p, sv, u, w, dx;
      float r_d = frad, u_d = 0.f, w_d = 0.f, p_d, s_d, dx_d;
      float alpha, gamma = 0.f, gamma_old, delta;
      // u = M^-1 r, w = -J u and both inner products (one reduction)
      auto precond_jvp = [&]() {
        MF_SUB(-1);
        const float gpart = precond_regs(r, u);
        MF_SUB(1);
        if (dyn) u_d = J_dd_inv * r_d;
        delta = jvp_regs(u, u_d, w, &w_d, gpart, &gamma);
        MF_SUB(2);
        if (tid == 0) MF_COUNT(3);
        if (dyn) gamma += r_d * u_d;
      };
      precond_jvp();
      alpha = gamma / (delta + 1e-30f);
#pragma unroll
      for (int k = 0; k < RF; ++k)
#pragma unroll
        for (int e = 0; e < RE; ++e) {
          p[k][e] = u[k][e];
          sv[k][e] = w[k][e];
          dx[k][e] = alpha * p[k][e];
          r[k][e] = r[k][e] - alpha * sv[k][e];
        }
      p_d = u_d;
      s_d = w_d;
      dx_d = alpha * p_d;
      r_d = r_d - alpha * s_d;
      for (int kk = 1; kk < n_cg; ++kk) {
        gamma_old = gamma;
        precond_jvp();
        const float beta = gamma / (gamma_old + 1e-30f);
        alpha = gamma / (delta - beta * gamma / alpha + 1e-30f);
#pragma unroll
        for (int k = 0; k < RF; ++k)
#pragma unroll
          for (int e = 0; e < RE; ++e) {
            p[k][e] = fmaf(beta, p[k][e], u[k][e]);
            sv[k][e] = fmaf(beta, sv[k][e], w[k][e]);
            dx[k][e] = fmaf(alpha, p[k][e], dx[k][e]);
            r[k][e] = r[k][e] - alpha * sv[k][e];
          }
        p_d = fmaf(beta, p_d, u_d);
        s_d = fmaf(beta, s_d, w_d);
        dx_d = fmaf(alpha, p_d, dx_d);
        r_d = r_d - alpha * s_d;
      }
      // x += dx with non-finite entries zeroed
      bad_local = 0;
#pragma unroll
      for (int k = 0; k < RF; ++k) {
        int base, n, f;
        bool thick;
        if (!slot(k, base, n, f, thick)) break;
        float* __restrict__ xs = s.x + base;
#pragma unroll
        for (int e = 0; e < RE; ++e) {
          const int j = lane * RE + e;
          if (j < n) {
            float v = dx[k][e];
            if (!isfinite(v)) { v = 0.f; bad_local = 1; }
            xs[j] = xs[j] + v;
          }
        }
      }
      if (dyn) {
        float v = dx_d;
        if (!isfinite(v)) v = 0.f;
        d = fmax_nan(d + v, 1.0f);
      }
      if (tid == 0) MF_COUNT(4);
    }
    resid = fmx;
    iters = it;
    if (!isfinite(fmx)) status |= MF_NONFINITE_BIT;
  }

  // ------------------------------------------------------------------
  // probability tables (built when (pCa, d) differ from the cached key)
  // ------------------------------------------------------------------
  __device__ void build_tables(float pCa, float d, bool sampling, bool absorbing) {
    build_tables_block(s.tab, pCa, d, sampling, sampling, absorbing, nullptr, 0, tid, NT);
  }
  // the tropomyosin tables alone (they do not depend on the spacing)
  __device__ void build_tm_tables(float pCa) {
    build_tables_block(s.tab, pCa, 0.f, true, false, false, nullptr, 0, tid, NT);
  }

  // Dynamic spacing rebuilds the crossbridge tables every step.  Only the
  // rows some head reads are built: the sampling keys of all heads (after
  // the tropomyosin update, thick_step's keys) or the absorbing keys of the
  // heads the metrics read (old state 2 or 3).  Flags and the key list
  // live in the CG vector pv, which is free outside the solve; the list is
  // in key order (neighbouring bins of one permissiveness share a warp, and
  // with them similar squaring counts: measured 0.5-1 % faster than a
  // bin-major list from the highest bin down).
  //
  // The absorbing rows of step t and the sampling rows of step t + 1 have
  // the same spacing (the one step t solved for) and, with pCa unchanged,
  // the same key: with merge_ok the absorbing build also builds every
  // sampling row when that takes fewer rounds of npairs matrices than the
  // absorbing rows now plus the sampling rows of the next step (estimated by
  // samp_est, the key count of the last sampling build; while the builds
  // merge, no sampling build runs and the estimate keeps the count that
  // started them).  Measured on 2x2 to 4x4 solved-spacing sweeps this beats
  // both separate builds of the read rows only (7-12 %) and a rule that
  // merges only when nearly every row is read.  Returns the key count of a
  // sampling build, or for an absorbing build 1 if every sampling row was
  // built with it, else 0.
  __device__ bool lazy_tables_fit() const {
    const int nk = A.pop.kx() * 2 * T.n_bins, nwords = (nk + 31) >> 5;
    return 4 * (nwords + 1) + 2 * nk <= 4 * T.n_dof;
  }
  __device__ int build_needed_tables(float pCa, float d, bool absorbing, bool merge_ok = false, int samp_est = 0) {
    const int kx = A.pop.kx(), nb = T.n_bins;
    const int nk = kx * 2 * nb, nwords = (nk + 31) >> 5, X = T.total_xbs;
    uint32_t* bits = reinterpret_cast<uint32_t*>(s.pv);
    int* count = reinterpret_cast<int*>(bits + nwords);
    int16_t* list = reinterpret_cast<int16_t*>(count + 1);
    __syncthreads();
    for (int w = tid; w < nwords; w += NT) bits[w] = 0u;
    __syncthreads();
    for (int i = tid; i < X; i += NT) {
      int key = -1;
      if (!absorbing) {
        key = sample_key(i);
      } else {
        const int so = s.old_xbs[i];
        if (so == 2 || so == 3) key = s.old_key[i];
      }
      if (key >= 0) atomicOr(&bits[key >> 5], 1u << (key & 31));
    }
    __syncthreads();
    if (warp == 0) {
      int base = 0;
      for (int c = 0; c < nwords; c += 32) {
        const int wi = c + lane;
        uint32_t wb = wi < nwords ? bits[wi] : 0u;
        const int n = __popc(wb);
        int incl = n;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int v = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += v;
        }
        int off = base + incl - n;
        while (wb) {
          list[off++] = (int16_t)(wi * 32 + __ffs(wb) - 1);
          wb &= wb - 1u;
        }
        base += __shfl_sync(0xffffffffu, incl, 31);
      }
      if (lane == 0) *count = base;
    }
    __syncthreads();
    const int nkeys = *count;
    constexpr int npairs = NT / 2;
    auto rounds = [](int n) { return (n + npairs - 1) / npairs; };
    const bool merge = absorbing && merge_ok && rounds(nk + nkeys) < rounds(nkeys) + rounds(samp_est);
    build_tables_block(s.tab, pCa, d, false, !absorbing || merge, absorbing, list, nkeys, tid, NT);
    __syncthreads();
    return absorbing ? (merge ? 1 : 0) : nkeys;
  }

  // ------------------------------------------------------------------
  // kinetics
  // ------------------------------------------------------------------
  // Nearest binding site of every head (kernels/geometry.py:60-262): the
  // first candidate of the head's face with the smallest |site - (crown + 13)|
  // among the valid ones (k < face_n, position > 0).  The candidate
  // positions of every face are staged once per step; on a face whose valid
  // candidates form one run of strictly monotone positions (the normal case:
  // sites along a filament) the argmin is found by bisection, with ties
  // resolved towards the lower index exactly as the linear scan does;
  // other faces use the linear scan over the staged positions.
  __device__ void nearest(float d) {
    const int X = T.total_xbs, W = T.width, nsi = T.n_sites, ntn = T.n_thick_nodes;
    const int nfaces = T.n_thin * 3;
    double* __restrict__ fp = s.face_pos;
    const int16_t* __restrict__ cands = T.face_sites;
    const uint8_t* __restrict__ fn = T.face_n;
    // one warp per face: its lanes stage the candidate positions and, on a
    // face of at most 32 candidates, classify the run from their own values
    for (int face = warp; face < nfaces; face += NW) {
      double pk = NAN;
      for (int k = lane; k < W; k += 32) {
        double pos = NAN;
        if (k < fn[face]) {
          const int g = (face / 3) * nsi + cands[face * W + k];
          pos = precise ? site_pos_d(g) : (double)s.x[ntn + g];
        }
        pos = pos > 0.0 ? pos : NAN;
        fp[face * W + k] = pos;
        if (W <= 32) pk = pos;
      }
      const bool v = pk == pk;
      const unsigned vm = __ballot_sync(0xffffffffu, v);
      const double pn = __shfl_down_sync(0xffffffffu, pk, 1);
      const bool pair = v && lane < 31 && ((vm >> (lane + 1)) & 1u);
      const unsigned pm = __ballot_sync(0xffffffffu, pair);
      const unsigned im = __ballot_sync(0xffffffffu, pair && pk < pn);
      const unsigned dm = __ballot_sync(0xffffffffu, pair && pk > pn);
      if (lane == 0) {
        int mono = 0, kl = 0, kh = 0;
        if (W <= 32) {
          if (vm == 0u) {
            mono = 3;  // no valid candidate: the scan keeps k = 0
          } else {
            kl = __ffs(vm) - 1;
            kh = 31 - __clz(vm);
            const int len = kh - kl + 1;
            const unsigned run = len == 32 ? 0xffffffffu : ((1u << len) - 1u);
            if ((vm >> kl) == run) mono = im == pm ? 1 : (dm == pm ? 2 : 0);
          }
        }
        s.face_mono[face] = (int8_t)mono;
        s.face_kl[face] = (int8_t)kl;
        s.face_kh[face] = (int8_t)kh;
      }
    }
    __syncthreads();
    for (int i = tid; i < X; i += NT) {
      const int face = T.xb_face[i];
      const int node = crown_node(i);
      const double* __restrict__ fpf = fp + face * W;
      const double head = precise ? crown_pos_d(node) + 13.0 : (double)(s.x[node] + 13.0f);
      auto dist = [&](int k) -> double {
        const double p = fpf[k];
        return precise ? fabs(p - head) : (double)fabsf((float)p - (float)head);
      };
      const int mono = s.face_mono[face];
      int bestk = 0;
      if (mono == 1 || mono == 2) {
        if (head == head) {
          const int kl = s.face_kl[face], kh = s.face_kh[face];
          int lo = kl, hi = kh + 1;
          while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            const double p = fpf[mid];
            const bool right = mono == 1 ? p >= head : p <= head;
            if (right) hi = mid;
            else lo = mid + 1;
          }
          if (lo > kl && (lo > kh || dist(lo - 1) <= dist(lo))) {
            bestk = lo - 1;
            while (bestk > kl && dist(bestk - 1) == dist(bestk)) --bestk;
          } else {
            bestk = lo;
          }
        }
      } else if (mono == 0) {
        double best = INFINITY;
        for (int k = 0; k < W; ++k) {
          const double p = fpf[k];
          if (p == p) {
            const double dd = dist(k);
            if (dd < best) { best = dd; bestk = k; }
          }
        }
      }
      const int site = cands[face * W + bestk];
      s.xb_near[i] = (int16_t)site;
      s.xb_ax[i] = xb_offset((face / 3) * nsi + site, node);
    }
    (void)d;
  }

  __device__ __forceinline__ float uniform_of(const uint32_t* key, int n, int i, const float* inj,
                                              size_t inj_off) const {
    if (inj) return inj[inj_off + i];
    return bits_to_uniform(bits32(part, key[0], key[1], (uint32_t)n, (uint32_t)i));
  }

  // after_loop: run by every thread once its sites are sampled, before the
  // update is published (work for threads with fewer sites)
  template <class Fn>
  __device__ void thin_step(const uint32_t* sub, size_t inj_off, Fn&& after_loop) {
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
        const int row = A.pop.kt() > 1 ? s.tlab[g] * 27 + cfg : cfg;
        const float* c = s.cum_tm + row * 16 + st * 4;
        ns = u < c[0] ? 0 : (u < c[1] ? 1 : (u < c[2] ? 2 : (u < c[3] ? 3 : 0)));
      }
      s.tm_new[g] = (int8_t)ns;
    }
    after_loop();
    __syncthreads();
    // the new states, and thick_step's empty bids per site (win1 / win2, in
    // the site region, which nothing reads between here and thick_step)
    int* win1 = reinterpret_cast<int*>(s.site);
    for (int g = tid; g < S; g += NT) {
      s.tm[g] = s.tm_new[g];
      win1[g] = -1;
      s.win2[g] = -1;
    }
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

  // Table key of head i at the current geometry: permissiveness of its
  // nearest site (tropomyosin state 3 and a valid head) and the bin of its
  // axial offset (transitions.py:807-922).
  __device__ __forceinline__ int sample_key(int i) const {
    const int nsi = T.n_sites;
    const int thin = thin_of(i);
    const int near = s.xb_near[i];
    const int site = near < 0 ? 0 : (near > nsi - 1 ? nsi - 1 : near);
    const bool perm = (s.tm[thin * nsi + site] == 3) && T.xb_valid[i];
    return pop_key(i) + (perm ? T.n_bins : 0) + bin_of(s.xb_ax[i]);
  }
  // first table key of head i's population (0 without per-population tables)
  __device__ __forceinline__ int pop_key(int i) const {
    return A.pop.kx() > 1 ? (int)s.xlab[i] * 2 * T.n_bins : 0;
  }

  __device__ void thick_step(const uint32_t* sub, size_t inj_off) {
    const int X = T.total_xbs, S = T.n_sites_total;
    const float* cum_xb = reinterpret_cast<const float*>(ws + L.cum_xb);
    int* win1 = reinterpret_cast<int*>(s.site);  // emptied by thin_step
    // sample, decide binding, and bid for the two scatter targets
    const int nsi = T.n_sites, nbins = T.n_bins;
    for (int i = tid; i < X; i += NT) {
      const int thin = thin_of(i);
      const int near = s.xb_near[i];
      const int site = near < 0 ? 0 : (near > nsi - 1 ? nsi - 1 : near);
      const int tgt = thin * nsi + site;
      const bool perm = (s.tm[tgt] == 3) && T.xb_valid[i];
      const int key = pop_key(i) + (perm ? nbins : 0) + bin_of(s.xb_ax[i]);
      s.xb_key[i] = (int16_t)key;
      const int old = s.xb_state[i];
      const float* c = cum_xb + key * 36 + old * 6;
      float cum[6];
#pragma unroll
      for (int k = 0; k < 6; ++k) cum[k] = __ldg(c + k);  // requested before the draw is computed
      const float u = uniform_of(sub, X, i, A.u_xb, inj_off);
      int ns = 0;
#pragma unroll
      for (int k = 5; k >= 0; --k)
        if (u < cum[k]) ns = k;
      const bool ob = old >= 1 && old <= 3, nbd = ns >= 1 && ns <= 3;
      const bool binding = !ob && nbd, unbinding = ob && !nbd;
      const bool occupied = s.thin_bound[tgt] >= 0;
      const bool can_bind = binding && perm && !occupied;
      const int ob_site = s.xb_bound[i];
      const int t1 = thin * nsi + (ob_site < 0 ? 0 : (ob_site > nsi - 1 ? nsi - 1 : ob_site));
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
