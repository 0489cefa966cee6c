// Shared host/device definitions: device lattice, per-condition workspace
// layout, Threefry-2x32, and the reduction-order helpers that reproduce the
// reference's jnp.cumsum / lax.associative_scan association.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define MF_HD __host__ __device__ __forceinline__

namespace mf {

#ifdef __CUDACC__
// max / min that return NaN when either operand is NaN, as jnp.maximum,
// jnp.minimum and jnp.clip do (fmaxf / fminf return the other operand), so
// that a NaN reaches the residual norm and the status bit the way it reaches
// the reference's while-loop test.  One instruction (PTX max.NaN / min.NaN,
// sm_80 and later).
__device__ __forceinline__ float fmax_nan(float a, float b) {
  float d;
  asm("max.NaN.f32 %0, %1, %2;" : "=f"(d) : "f"(a), "f"(b));
  return d;
}
__device__ __forceinline__ float fmin_nan(float a, float b) {
  float d;
  asm("min.NaN.f32 %0, %1, %2;" : "=f"(d) : "f"(a), "f"(b));
  return d;
}
#endif

constexpr int kNParams = 44;
constexpr int kNMetrics = 52;
// per-warp partials of the metrics' fused block reduction (one per lane)
constexpr int kRedPartials = 32;
// filaments per warp of the register-resident precise CG at nt threads
__host__ __device__ constexpr int regcg_rf(int nt) { return nt == 384 ? 1 : (nt == 512 ? 3 : 2); }
constexpr int kMaxLevels = 12;

// DynamicParams field indices (reference core/params.py:73-556 order).
enum P : int {
  THICK_K = 0, THIN_K, XB_C_REST_WEAK, XB_C_REST_STRONG, XB_C_K_WEAK, XB_C_K_STRONG,
  XB_G_REST_WEAK, XB_G_REST_STRONG, XB_G_K_WEAK, XB_G_K_STRONG, TITIN_A, TITIN_B, TITIN_REST,
  TM_K_01, TM_K_12, TM_K_23, TM_K_30, TM_KEQ_01, TM_KEQ_12, TM_KEQ_23, TM_J_C, TM_J_M,
  XB_R01_COEFF, XB_R12_COEFF, XB_R23_COEFF, XB_R34_COEFF, XB_DELTA_23, XB_DELTA_34, XB_R40,
  XB_R04, XB_R05, XB_U_DRX, XB_U_LOOSE, XB_U_TIGHT_1, XB_U_TIGHT_2, XB_SRX_K0, XB_SRX_KMAX,
  XB_SRX_B, XB_SRX_CA50, TEMP_CELSIUS, SOLVER_TOL, PCA, Z_LINE, LATTICE_SPACING
};

// Metric slots (reference metrics_fn.py:343-417 key order).
enum M : int {
  M_AXIAL_FORCE = 0, M_SOLVER_RESIDUAL, M_Z_LINE, M_PCA, M_LATTICE_SPACING, M_N_BOUND,
  M_N_XB_DRX, M_N_XB_LOOSE, M_N_XB_TIGHT_1, M_N_XB_TIGHT_2, M_N_XB_FREE_2, M_N_XB_SRX,
  M_FRAC_XB_BOUND, M_FRAC_XB_DRX, M_FRAC_XB_LOOSE, M_FRAC_XB_TIGHT_1, M_FRAC_XB_TIGHT_2,
  M_FRAC_XB_FREE_2, M_FRAC_XB_SRX, M_N_TM_0, M_N_TM_1, M_N_TM_2, M_N_TM_3, M_FRAC_TM_0,
  M_FRAC_TM_1, M_FRAC_TM_2, M_FRAC_TM_3, M_ACTIN_PERM, M_FRAC_TM_2_OV, M_FRAC_TM_3_OV,
  M_FRAC_TM_AVAIL_OV, M_N_OVERLAP, M_ATP_CONSUMED, M_NEWLY_BOUND, M_THICK_D_MEAN, M_THICK_D_MAX,
  M_THICK_D_MIN, M_THICK_D_STD, M_THIN_D_MEAN, M_THIN_D_MAX, M_THIN_D_MIN, M_THIN_D_STD,
  M_THICK_E_AVG, M_THICK_E_DELTA, M_TITIN_E_AVG, M_TITIN_E_DELTA, M_WORK_THICK,
  M_WORK_THICK_MEAN, M_ATP_EXPECTED_P, M_XB_TEAR, M_WORK_PER_ATP, M_NEWTON_ITERS
};

// Down-sweep level structure of lax.associative_scan for a length-n scan:
// n_0 = n, n_{l+1} = floor(n_l / 2) while n_l >= 2.  Level l occupies
// [off[l], off[l] + len[l]) of a scratch array.
struct ScanPlan {
  int n, levels, total;
  int len[kMaxLevels];
  int off[kMaxLevels];
};

MF_HD ScanPlan make_scan_plan(int n) {
  ScanPlan p{};
  p.n = n;
  int l = 0, off = 0, m = n;
  while (true) {
    p.len[l] = m;
    p.off[l] = off;
    off += m;
    ++l;
    if (m < 2 || l >= kMaxLevels) break;
    m = m / 2;
  }
  p.levels = l;
  p.total = off;
  return p;
}

// Lattice as the kernels read it (one copy per topology, global memory).
struct TopoDev {
  int n_thick, n_crowns, n_thin, n_sites, nxb, width, n_bins;
  int total_xbs, n_dof, n_sites_total, n_thick_nodes;
  float crown_min, crown_max;
  ScanPlan plan_thick, plan_thin;
  const int16_t* xb_face;    // [X]  thin*3 + face of each head's target
  const uint8_t* xb_valid;   // [X]
  const int16_t* face_sites; // [n_thin*3*width] candidate sites, padded like xb_to_site_indices
  const uint8_t* face_n;     // [n_thin*3] valid candidates per face
  const int16_t* tm_prev;    // [S] same-chain predecessor (local index)
  const int16_t* tm_next;    // [S]
  const float* crown_off;    // [n_thick*n_crowns]
  const float* crown_rest;
  const float* bind_off;     // [S]
  const float* bind_rest;
  const float* thin_cum;     // [S]
  const float* edges;        // [n_bins+1]
  const float* centers;      // [n_bins]
  // precise-mode spring prestrain constants, rounded from float64
  const float* thick_c;      // [n_thick*n_crowns]: off[c]-off[c-1]-rest[c]
  const float* thin_c;       // [S]: off[j]-off[j+1]-rest[j], last: off-rest
};

// Longest filament the kernels take (nodes), and the per-warp scan reversal
// buffer of a lattice: 128 floats up to 128 nodes, else 256.
constexpr int kMaxFilament = 256;
constexpr int kWideThreads = 512;  // smallest CTA size for filaments of more than 128 nodes
MF_HD int max_filament(const TopoDev& t) { return t.n_crowns > t.n_sites ? t.n_crowns : t.n_sites; }
MF_HD int scan_cap(const TopoDev& t) { return max_filament(t) <= 128 ? 128 : 256; }

// Byte layout of one condition's resident workspace (global memory).
struct SlotLayout {
  size_t x, xb_state, xb_bound, xb_near, xb_ax, xb_key, tm, thin_bound, misc, cum_xb, pabs, cum_tm,
      coef, vec, total;
};

MF_HD size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Subpopulations of a batch (reference core/subpopulation.py): K populations,
// flag bits POP_EXPLICIT (labels select a population's tables; else the K
// generators are blended), POP_XB / POP_TM (the rate families they change).
// K <= 1 is a single population.
constexpr int POP_EXPLICIT = 1, POP_XB = 2, POP_TM = 4, kMaxPops = 4;
struct PopShape {
  int K = 1;
  int flags = 0;
  // crossbridge / tropomyosin table sets kept per condition
  MF_HD int kx() const { return (K > 1 && (flags & (POP_EXPLICIT | POP_XB)) == (POP_EXPLICIT | POP_XB)) ? K : 1; }
  MF_HD int kt() const { return (K > 1 && (flags & (POP_EXPLICIT | POP_TM)) == (POP_EXPLICIT | POP_TM)) ? K : 1; }
  // blended (mean-field) generators of a family
  MF_HD bool blend_xb() const { return K > 1 && (flags & (POP_EXPLICIT | POP_XB)) == POP_XB; }
  MF_HD bool blend_tm() const { return K > 1 && (flags & (POP_EXPLICIT | POP_TM)) == POP_TM; }
  // the population rows are read at all
  MF_HD bool active() const { return K > 1 && (flags & (POP_XB | POP_TM)) != 0; }
};

MF_HD SlotLayout slot_layout(int n_dof, int X, int S, int n_bins, int coef_floats, int kx = 1, int kt = 1) {
  SlotLayout L{};
  size_t o = 0;
  L.x = o; o = align_up(o + sizeof(float) * n_dof, 16);
  L.xb_state = o; o = align_up(o + X, 16);
  L.xb_bound = o; o = align_up(o + 2 * X, 16);
  L.xb_near = o; o = align_up(o + 2 * X, 16);
  L.xb_ax = o; o = align_up(o + 4 * X, 16);
  L.xb_key = o; o = align_up(o + 2 * X, 16);
  L.tm = o; o = align_up(o + S, 16);
  L.thin_bound = o; o = align_up(o + 2 * S, 16);
  L.misc = o; o = align_up(o + 64 * sizeof(double), 16);
  L.cum_xb = o; o = align_up(o + sizeof(float) * kx * 2 * n_bins * 36, 16);
  L.pabs = o; o = align_up(o + sizeof(float) * kx * 2 * n_bins * 3, 16);
  L.cum_tm = o; o = align_up(o + sizeof(float) * kt * 27 * 16, 16);
  L.coef = o; o = align_up(o + sizeof(float) * coef_floats, 16);
  L.vec = o; o = align_up(o + sizeof(float) * (7 * n_dof + 4 * X), 16);  // CG vectors + head terms when not in smem
  L.total = align_up(o, 256);
  return L;
}

// Slots of the per-condition misc block (doubles).
enum Misc : int {
  MS_KEY = 0,          // uint32 pair stored in a double slot
  MS_CUR_LS = 1,       // carried lattice spacing
  MS_ZREF = 2,         // precise mode: z of the thin reference positions
  MS_TAB_PCA = 3,      // cache key of the sampling tables
  MS_TAB_D = 4,
  MS_ABS_PCA = 5,      // cache key of the absorbing table
  MS_ABS_D = 6,
  MS_STATUS = 7,
  MS_T_DONE = 8,
  MS_L0 = 9,           // z at step 0 (Poisson reference)
};

// ---------------------------------------------------------------------------
// Threefry-2x32, 20 rounds (Salmon et al., SC'11), and the jax.random layering.
// ---------------------------------------------------------------------------
MF_HD uint32_t rotl32(uint32_t v, int r) { return (v << r) | (v >> (32 - r)); }

MF_HD void threefry2x32(uint32_t k0, uint32_t k1, uint32_t x0, uint32_t x1, uint32_t& y0,
                        uint32_t& y1) {
  const uint32_t ks2 = k0 ^ k1 ^ 0x1BD11BDAu;
  const uint32_t ks[3] = {k0, k1, ks2};
  uint32_t a = x0 + k0, b = x1 + k1;
#define MF_R(r) a += b; b = rotl32(b, r); b ^= a;
  MF_R(13) MF_R(15) MF_R(26) MF_R(6)  a += ks[1]; b += ks[2] + 1u;
  MF_R(17) MF_R(29) MF_R(16) MF_R(24) a += ks[2]; b += ks[0] + 2u;
  MF_R(13) MF_R(15) MF_R(26) MF_R(6)  a += ks[0]; b += ks[1] + 3u;
  MF_R(17) MF_R(29) MF_R(16) MF_R(24) a += ks[1]; b += ks[2] + 4u;
  MF_R(13) MF_R(15) MF_R(26) MF_R(6)  a += ks[2]; b += ks[0] + 5u;
#undef MF_R
  y0 = a;
  y1 = b;
}

// split(key, num)[i] in the partitionable layout: H(key, (0, i)).
MF_HD void split_part(uint32_t k0, uint32_t k1, uint32_t i, uint32_t& o0, uint32_t& o1) {
  threefry2x32(k0, k1, 0u, i, o0, o1);
}

// split(key, num)[i] in the original layout: counters iota(2n) cut in halves.
MF_HD void split_orig(uint32_t k0, uint32_t k1, uint32_t num, uint32_t i, uint32_t& o0,
                      uint32_t& o1) {
  // flat = concat(H(x0=c[:n], x1=c[n:]).y0, .y1); key i = (flat[2i], flat[2i+1])
  uint32_t out[2];
  for (int w = 0; w < 2; ++w) {
    uint32_t f = 2u * i + (uint32_t)w;  // index into flat (length 2n)
    uint32_t pair = f < num ? f : f - num;
    uint32_t y0, y1;
    threefry2x32(k0, k1, pair, pair + num, y0, y1);
    out[w] = f < num ? y0 : y1;
  }
  o0 = out[0];
  o1 = out[1];
}

MF_HD void split2(bool part, uint32_t k0, uint32_t k1, uint32_t i, uint32_t& o0, uint32_t& o1) {
  if (part) split_part(k0, k1, i, o0, o1);
  else split_orig(k0, k1, 2u, i, o0, o1);
}

// random_bits(key, (n,))[i], 32-bit.
MF_HD uint32_t bits32(bool part, uint32_t k0, uint32_t k1, uint32_t n, uint32_t i) {
  uint32_t y0, y1;
  if (part) {
    threefry2x32(k0, k1, 0u, i, y0, y1);
    return y0 ^ y1;
  }
  uint32_t h = (n + 1u) / 2u;  // odd n is padded with a zero counter
  uint32_t pair = i < h ? i : i - h;
  uint32_t c1 = pair + h;
  if (c1 >= n) c1 = 0u;  // the padding counter
  threefry2x32(k0, k1, pair, c1, y0, y1);
  return i < h ? y0 : y1;
}

MF_HD float bits_to_uniform(uint32_t b) {
  uint32_t fb = (b >> 9) | 0x3F800000u;
  float f;
#ifdef __CUDA_ARCH__
  f = __uint_as_float(fb);
#else
  __builtin_memcpy(&f, &fb, 4);
#endif
  f = f - 1.0f;
  return f < 0.0f ? 0.0f : f;
}

// The four per-step splits of timestep.py:120,125 and transitions.py:615,1160:
// k, thin_k = split(k); _, sub_thin = split(thin_k)
// k, thick_k = split(k); _, sub_thick = split(thick_k)
MF_HD void step_keys(bool part, uint32_t k0, uint32_t k1, uint32_t* sub_thin, uint32_t* sub_thick,
                     uint32_t* k_next) {
  uint32_t a0, a1, t0, t1;
  split2(part, k0, k1, 0u, a0, a1);
  split2(part, k0, k1, 1u, t0, t1);
  split2(part, t0, t1, 1u, sub_thin[0], sub_thin[1]);
  uint32_t b0, b1, h0, h1;
  split2(part, a0, a1, 0u, b0, b1);
  split2(part, a0, a1, 1u, h0, h1);
  split2(part, h0, h1, 1u, sub_thick[0], sub_thick[1]);
  k_next[0] = b0;
  k_next[1] = b1;
}

}  // namespace mf
