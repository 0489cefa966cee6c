// Kernel body: per-CTA set-up, the initial equilibrium, the step loop and the
// fused metrics epilogue.  See mf_step.cuh for the per-phase device code.
#pragma once
#include "mf_step.cuh"

namespace mf {

// Static shared memory of the kernel (the CTA-shared lattice, carve and
// condition structs of run_condition, about 1 KB) plus headroom; the dynamic
// carve below must fit in the opt-in limit next to it.
constexpr size_t kStaticSmem = 2048;

// One region holds three phase-disjoint uses: the per-site scatter words of
// the kinetics step (site = win1, then win2), the staged candidate positions
// of the nearest-site search (face_pos, doubles, over both), and from the
// bound-head list through the solve the per-site head pairs (site_h, over
// site) next to the per-site head counts (win2).
__host__ __device__ inline size_t site_region_bytes(const TopoDev& t) {
  const size_t words = 8 * (size_t)t.n_sites_total;
  const size_t faces = sizeof(double) * (size_t)t.n_thin * 3 * t.width;
  return words > faces ? words : faces;
}

// Shared-memory bytes needed by one condition of this lattice with NT threads.
// Reduction scratch: 32 partials per warp (the metrics' fused reduction),
// two double-buffered 96-float slots for the one-barrier reductions, and the
// force broadcast.
__host__ __device__ constexpr int red_floats(int nw) { return kRedPartials * nw + 2 * 96 + 1; }

// Where the CG vectors and head terms of a condition live (kernel flag bits
// 64 and 128).  LAYOUT_SMEM: all in shared memory; LAYOUT_GLOBAL: in the
// workspace (lattices too large for shared memory); LAYOUT_REGS: the
// register-resident CG, which keeps only x and u in shared memory.
enum Layout { LAYOUT_SMEM = 0, LAYOUT_GLOBAL = 1, LAYOUT_REGS = 2 };
constexpr int FLAG_VEC_GLOBAL = 64, FLAG_REGS = 128;

// Whether the register-resident precise CG covers this lattice at nt threads
// (regcg_rf filaments per warp, 3 nodes per lane, crowns of 3 heads).
__host__ __device__ inline bool regcg_fits(const TopoDev& t, int nt) {
  const int rf = regcg_rf(nt), re = 3;
  return t.n_thick + t.n_thin <= rf * (nt / 32) && t.n_crowns <= 32 * re && t.n_sites <= 32 * re && t.nxb == 3;
}

// Shared-memory bytes of one condition of this lattice with nt threads in one
// precision mode, layout and spacing mode (mirrors carve() below: every array
// both modes use, plus the float32 scan-reversal buffers or the precise-mode
// CG vectors w and s, and the per-head spacing derivatives when dyn).
__host__ __device__ inline size_t smem_bytes(const TopoDev& t, int nt, int layout, bool precise, bool dyn,
                                             PopShape pop = PopShape()) {
  const bool vec_global = layout == LAYOUT_GLOBAL;
  const int N = t.n_dof, X = t.total_xbs, S = t.n_sites_total;
  const int nw = nt / 32;
  const CoefLayout cl = coef_layout(t);
  size_t o = 0;
  auto add = [&](size_t bytes) { o = align_up(o + bytes, 16); };
  add(sizeof(double) * 64);                // redd
  add(sizeof(float) * red_floats(nw));     // red
  if (layout == LAYOUT_REGS) add(sizeof(float) * 2 * N);  // x zz
  else if (!vec_global) add(sizeof(float) * (precise ? 7 : 5) * N);  // x r dx pv zz (+ wv sv)
  if (!vec_global) add(sizeof(float) * (dyn ? 4 : 2) * X);  // fxb fdx (+ fdd frdd)
  add(sizeof(float) * X);                  // xb_ax
  add(site_region_bytes(t));               // site / win1 | win2, overlaid by face_pos and site_h
  add(sizeof(int16_t) * 2 * X);            // xb_bound xb_near
  add(sizeof(int16_t) * S);                // thin_bound
  add(X);                                  // xb_state
  add(2 * S);                              // tm tm_new
  add(sizeof(float) * pop.kt() * 27 * 16);  // cum_tm
  add(sizeof(float) * pop.kx() * 6 * t.n_bins);  // pabs
  add(sizeof(float) * cl.total);           // coef
  if (!precise) add(sizeof(float) * nw * scan_cap(t));  // scan reversal buffer per warp
  add(sizeof(float) * kNParams);           // P
  add(sizeof(float) * 4 * t.n_thick);      // tvec
  add(sizeof(int16_t) * X);                // blist
  add(sizeof(int) * 4);                    // nbound
  add(sizeof(int) * 32);                   // wsum
  add(sizeof(int16_t) * X);                // xb_key
  add(sizeof(int) * X);                    // hsite
  add(3 * t.n_thin * 3);                   // face_mono face_kl face_kh
  if (!vec_global) {                       // old-state snapshot
    add(sizeof(float) * t.n_thick_nodes);
    add(X);
    add(sizeof(int16_t) * X);
  }
  if (pop.active()) {                      // population rows, fractions, labels
    add(sizeof(float) * pop.K * kNParams);
    add(sizeof(float) * pop.K);
    if (pop.kx() > 1) add(X);
    if (pop.kt() > 1) add(S);
  }
  return o;
}

template <int NT, bool PR, bool DY>
__device__ void carve(Sim<NT, PR, DY>& m, char* base, int layout) {
  const TopoDev& t = m.T;
  const int N = t.n_dof, X = t.total_xbs, S = t.n_sites_total;
  const bool vec_global = layout == LAYOUT_GLOBAL;
  size_t o = 0;
  auto take = [&](size_t bytes) { char* p = base + o; o = align_up(o + bytes, 16); return p; };
  m.s.redd = (double*)take(sizeof(double) * 64);
  m.s.red = (float*)take(sizeof(float) * red_floats(NT / 32));
  // the workspace keeps room for all seven vectors; shared memory only for
  // the ones this mode uses
  if (layout == LAYOUT_REGS) {
    float* v2 = (float*)take(sizeof(float) * 2 * N);
    m.s.x = v2;
    m.s.zz = v2 + N;
    m.s.r = m.s.dx = m.s.wv = m.s.sv = nullptr;
    m.s.pv = m.s.zz;  // only the table-key list uses pv outside a smem CG; u is free then
  } else {
    float* v7 = vec_global ? reinterpret_cast<float*>(m.ws + m.L.vec) : (float*)take(sizeof(float) * (PR ? 7 : 5) * N);
    m.s.x = v7; m.s.r = v7 + N; m.s.dx = v7 + 2 * N; m.s.pv = v7 + 3 * N; m.s.zz = v7 + 4 * N;
    m.s.wv = PR ? v7 + 5 * N : nullptr;
    m.s.sv = PR ? v7 + 6 * N : nullptr;
  }
  // fxb fdx, and fdd frdd only in dynamic-spacing kernels (the workspace keeps room for all four)
  float* f4 = vec_global ? reinterpret_cast<float*>(m.ws + m.L.vec) + 7 * N : (float*)take(sizeof(float) * (DY ? 4 : 2) * X);
  m.s.fxb = f4; m.s.fdx = f4 + X;
  m.s.fdd = (DY || vec_global) ? f4 + 2 * X : nullptr;
  m.s.frdd = (DY || vec_global) ? f4 + 3 * X : nullptr;
  m.s.xb_ax = (float*)take(sizeof(float) * X);
  {
    char* reg = take(site_region_bytes(t));
    m.s.site = (float*)reg;
    m.s.win2 = (int*)(reg + sizeof(float) * S);
    m.s.face_pos = (double*)reg;
    m.s.site_h = (int16_t*)reg;  // 2S int16 = the bytes of site
  }
  int16_t* i2 = (int16_t*)take(sizeof(int16_t) * 2 * X);
  m.s.xb_bound = i2; m.s.xb_near = i2 + X;
  m.s.thin_bound = (int16_t*)take(sizeof(int16_t) * S);
  m.s.xb_state = (int8_t*)take(X);
  int8_t* t2 = (int8_t*)take(2 * S);
  m.s.tm = t2; m.s.tm_new = t2 + S;
  const PopShape& pop = m.A.pop;
  m.s.cum_tm = (float*)take(sizeof(float) * pop.kt() * 27 * 16);
  m.s.pabs = (float*)take(sizeof(float) * pop.kx() * 6 * t.n_bins);
  m.s.coef = (float*)take(sizeof(float) * m.cl.total);
  m.s.scan = PR ? nullptr : (float*)take(sizeof(float) * NT / 32 * scan_cap(t));
  m.s.P = (float*)take(sizeof(float) * kNParams);
  m.s.tvec = (float*)take(sizeof(float) * 4 * t.n_thick);
  m.s.blist = (int16_t*)take(sizeof(int16_t) * X);
  m.s.nbound = (int*)take(sizeof(int) * 4);
  m.s.wsum = (int*)take(sizeof(int) * 32);
  m.s.xb_key = (int16_t*)take(sizeof(int16_t) * X);
  m.s.hsite = (int*)take(sizeof(int) * X);
  m.s.face_mono = (int8_t*)take(3 * t.n_thin * 3);
  m.s.face_kl = m.s.face_mono + t.n_thin * 3;
  m.s.face_kh = m.s.face_kl + t.n_thin * 3;
  if (!vec_global) {
    m.s.old_thick = (float*)take(sizeof(float) * t.n_thick_nodes);
    m.s.old_xbs = (int8_t*)take(X);
    m.s.old_key = (int16_t*)take(sizeof(int16_t) * X);
  } else {
    // the persisted copies are only rewritten at the end of a launch, so
    // they double as snapshot space meanwhile
    m.s.old_thick = reinterpret_cast<float*>(m.ws + m.L.x);
    m.s.old_xbs = reinterpret_cast<int8_t*>(m.ws + m.L.xb_state);
    m.s.old_key = reinterpret_cast<int16_t*>(m.ws + m.L.xb_near);
  }
  m.s.Pk = m.s.fk = nullptr;
  m.s.xlab = m.s.tlab = nullptr;
  if (pop.active()) {
    m.s.Pk = (float*)take(sizeof(float) * pop.K * kNParams);
    m.s.fk = (float*)take(sizeof(float) * pop.K);
    if (pop.kx() > 1) m.s.xlab = (int8_t*)take(X);
    if (pop.kt() > 1) m.s.tlab = (int8_t*)take(S);
  }
  // the table builder's inputs (the timestep is set by the caller)
  TableCtx& tc = m.s.tab;
  tc.P = m.s.P;
  tc.centers = t.centers;
  tc.nb = t.n_bins;
  tc.sq64 = m.A.sq64_from;
  tc.cum_tm = m.s.cum_tm;
  tc.cum_xb = reinterpret_cast<float*>(m.ws + m.L.cum_xb);
  tc.pabs = m.s.pabs;
  tc.pop = pop;
  tc.Pk = m.s.Pk;
  tc.fk = m.s.fk;
}

// ---------------------------------------------------------------------------
// metrics epilogue (metrics_fn.py:154-417), written to metrics[b][k][t]
// ---------------------------------------------------------------------------
// Every thread accumulates its share of the 31 block totals (counts, sums,
// extrema and the thick-filament energies), the warps reduce them with one
// transposed exchange and meet at a single barrier.  After it every warp
// forms the totals from the per-warp partials and stores its share of the
// 18 output groups (group q = lane * NW + warp), so no warp carries the
// whole epilogue.  The axial force is summed in filament order by one thread
// during the partial pass and handed over through the same barrier.
template <int NT, bool PR, bool DY>
__device__ void metrics(Sim<NT, PR, DY>& m, int t, float zl, float pCa, float new_ls, double resid, int iters,
                        float* Mo) {
  const TopoDev& T = m.T;
  const int X = T.total_xbs, S = T.n_sites_total, NTN = T.n_thick_nodes;
  const int tid = m.tid;
  constexpr int NW = NT / 32;
  const int lane = m.lane, warp = m.warp;
  const float* pabs = m.s.pabs;
  const float* old_x = m.s.old_thick;
  const float* P = m.s.P;
  float* red = m.s.red;
  float* force_slot = red + red_floats(NW) - 1;
#ifdef MF_PHASE_TIMING
  // diagnostic build only: thread 0's own timeline through the epilogue
  long long mt0 = clock64();
#define MF_MT(k)                                       \
  do {                                                 \
    if (tid == 0) {                                    \
      const long long now_ = clock64();                \
      m.sub_acc[8 + (k)] += (double)(now_ - mt0);      \
      mt0 = now_;                                      \
    }                                                  \
  } while (0)
#else
#define MF_MT(k) do { } while (0)
#endif
  if (tid == NT - 1 - T.n_thick) {
    // axial force: sum over thick filaments in filament order, on a thread
    // with the lightest share of the loops below (the energies take the
    // last n_thick threads)
    float force = 0.f;
    for (int th = 0; th < T.n_thick; ++th) {
      const int n0 = th * T.n_crowns;
      const float u = m.precise ? m.s.x[n0] : m.s.x[n0] - T.crown_off[n0];
      force += u * P[THICK_K];
    }
    *force_slot = force;
  }
  // per-thread partials: counts (exact in float), sums, extrema
  float c_xb[7] = {0, 0, 0, 0, 0, 0, 0};  // 6 states + bound
  float c_tm[4] = {0, 0, 0, 0};
  float ov = 0.f, ov2 = 0.f, ov3 = 0.f, atp = 0.f, newly = 0.f, atp_p = 0.f, tear = 0.f;
  const float near_b = T.crown_min - 13.0f, far_b = T.crown_max + 13.0f;
  for (int i = tid; i < X; i += NT) {
    const int sn = m.s.xb_state[i], so = m.s.old_xbs[i];
#pragma unroll
    for (int k = 0; k < 6; ++k) c_xb[k] += (sn == k);  // compile-time indices keep the counts in registers
    c_xb[6] += (sn >= 1 && sn <= 3);
    atp += (so == 3) && (sn == 4 || sn == 0);
    newly += (so == 0) && (sn == 1);
    if (so == 2 || so == 3) {
      // expected exits from the absorbing generator at the pre-step geometry
      // (metrics_fn.py:297-338); its table row is the one sampled last step
      const int key = m.s.old_key[i];
      if (so == 3) atp_p += pabs[key * 3 + 0];
      tear += pabs[key * 3 + (so == 2 ? 1 : 2)];
    }
  }
  // displacement statistics: one pass around a provisional shift (the first
  // node), var = E[(x-s)^2] - (E[x]-s)^2 with s near the mean
  const float t_shift = m.precise ? m.s.x[0] : m.s.x[0] - T.crown_off[0];
  float n_shift;
  if (!m.precise) n_shift = m.s.x[NTN] - T.thin_cum[0];
  else n_shift = (float)((m.zref - (double)T.bind_off[0]) + (double)m.s.x[NTN] - (double)T.thin_cum[0]);
  float tsum = 0.f, tsq = 0.f, nsum = 0.f, nsq = 0.f, dxs = 0.f;
  float tmin = INFINITY, tmax = -INFINITY, nmin = INFINITY, nmax = -INFINITY;
  for (int i = tid; i < NTN; i += NT) {
    const float dsp = m.precise ? m.s.x[i] : m.s.x[i] - T.crown_off[i];
    const float c = dsp - t_shift;
    tsum += c;
    tsq = fmaf(c, c, tsq);
    tmin = fmin_nan(tmin, dsp);
    tmax = fmax_nan(tmax, dsp);
    dxs += m.s.x[i] - old_x[i];
  }
  for (int g = tid; g < S; g += NT) {
    const int st = m.s.tm[g];
#pragma unroll
    for (int k = 0; k < 4; ++k) c_tm[k] += (st == k);
    float xa, dsp;
    if (!m.precise) {
      xa = m.s.x[NTN + g];
      dsp = xa - T.thin_cum[g];
    } else {
      const double xd = (m.zref - (double)T.bind_off[g]) + (double)m.s.x[NTN + g];
      xa = (float)xd;
      dsp = (float)(xd - (double)T.thin_cum[g]);
    }
    const bool o = xa >= near_b && xa <= far_b && xa > 0.0f;
    ov += o;
    ov2 += o && st == 2;
    ov3 += o && st == 3;
    const float c = dsp - n_shift;
    nsum += c;
    nsq = fmaf(c, c, nsq);
    nmin = fmin_nan(nmin, dsp);
    nmax = fmax_nan(nmax, dsp);
  }
  // energies of the thick backbone's first spring and of titin
  // (metrics_fn.py:262-288), one filament per thread counted from the last
  // thread (the first threads carry the force sum and the loop remainders)
  float e_new = 0.f, e_delta = 0.f, te_new = 0.f, te_delta = 0.f;
  {
    const float k = P[THICK_K];
    const float a = P[TITIN_A], bb = P[TITIN_B], r0 = P[TITIN_REST];
    for (int th = NT - 1 - tid; th < T.n_thick; th += NT) {
      const int n0 = th * T.n_crowns;
      const float u_new = m.precise ? m.s.x[n0] : m.s.x[n0] - T.crown_off[n0];
      const float u_old = m.precise ? old_x[n0] : old_x[n0] - T.crown_off[n0];
      const float en = 0.5f * k * (u_new * u_new);
      const float eo = 0.5f * k * (u_old * u_old);
      e_new += en;
      e_delta += en - eo;
      const int nl = n0 + T.n_crowns - 1;
      float ad_new, ad_old;
      if (!m.precise) {
        ad_new = zl - m.s.x[nl];
        ad_old = zl - old_x[nl];
      } else {
        const float zc = (float)((double)zl - (double)T.crown_off[nl]);
        ad_new = zc - m.s.x[nl];
        ad_old = zc - old_x[nl];
      }
      const float Ln = sqrtf(ad_new * ad_new + new_ls * new_ls);
      const float Lo = sqrtf(ad_old * ad_old + new_ls * new_ls);
      const float tn = (a / bb) * (expf(bb * (Ln - r0)) - 1.0f);
      const float to = (a / bb) * (expf(bb * (Lo - r0)) - 1.0f);
      te_new += tn;
      te_delta += tn - to;
    }
  }
  MF_MT(0);
  // values 0-3 are maxima (minima negated), the rest sums
  float r[32] = {-tmin, tmax, -nmin, nmax,
                 c_xb[0], c_xb[1], c_xb[2], c_xb[3], c_xb[4], c_xb[5], c_xb[6],
                 c_tm[0], c_tm[1], c_tm[2], c_tm[3], ov, ov2, ov3, atp, newly,
                 tsum, tsq, nsum, nsq, dxs, atp_p, tear, e_new, e_delta, te_new, te_delta, 0.f};
  red[warp * 32 + lane] = warp_reduce_transposed<4>(r, lane);  // warp-major: no bank conflicts
  MF_MT(1);
  __syncthreads();
  MF_MT(2);
  // block totals, lane k holding total k (every warp forms them itself)
  float R = red[lane];
#pragma unroll 4
  for (int w = 1; w < NW; ++w) R = lane < 4 ? fmax_nan(R, red[w * 32 + lane]) : R + red[w * 32 + lane];
  const float force = *force_slot;
  auto tot = [&](int k) { return __shfl_sync(0xffffffffu, R, k); };
  MF_MT(3);
  const int q = lane * NW + warp;  // this lane's output group
  // every shuffle is executed by all 32 lanes; the branches below only store
  const float own = tot(q < 6 ? 4 + q : (q < 10 ? 5 + q : 14));
  const float tmin_ = -tot(0), tmax_ = tot(1), nmin_ = -tot(2), nmax_ = tot(3);
  const float nb = tot(10), nov = tot(15), n2 = tot(16), n3 = tot(17);
  const float r18 = tot(18), r19 = tot(19), r20 = tot(20), r21 = tot(21), r22 = tot(22), r23 = tot(23);
  const float r24 = tot(24), r25 = tot(25), r26 = tot(26);
  const float en_new = tot(27), en_delta = tot(28), ten_new = tot(29), ten_delta = tot(30);
  MF_MT(4);
  const float nx = (float)X, nt = (float)S;
  auto put = [&](int k, float v) { Mo[(size_t)k * m.Tstride + t] = v; };
  if (q < 6) {
    put(M_N_XB_DRX + q, own);
    put(M_FRAC_XB_DRX + q, own / nx);
  } else if (q < 10) {
    const int j = q - 6;
    put(M_N_TM_0 + j, own);
    put(M_FRAC_TM_0 + j, own / nt);
  } else if (q == 10) {
    put(M_AXIAL_FORCE, force);
    put(M_SOLVER_RESIDUAL, (float)resid);
    put(M_Z_LINE, zl);
    put(M_PCA, pCa);
    put(M_LATTICE_SPACING, new_ls);
  } else if (q == 11) {
    put(M_N_BOUND, nb);
    put(M_FRAC_XB_BOUND, nb / nx);
    put(M_ACTIN_PERM, own / nt);
  } else if (q == 12) {
    put(M_FRAC_TM_2_OV, n2 / nov);
    put(M_FRAC_TM_3_OV, n3 / nov);
    put(M_FRAC_TM_AVAIL_OV, (n2 + n3) / nov);
    put(M_N_OVERLAP, nov);
  } else if (q == 13) {
    put(M_ATP_CONSUMED, r18);
    put(M_NEWLY_BOUND, r19);
    put(M_ATP_EXPECTED_P, r25);
    put(M_XB_TEAR, r26);
    put(M_NEWTON_ITERS, (float)iters);
  } else if (q == 14) {
    const float tmean_c = r20 / (float)NTN;
    put(M_THICK_D_MEAN, t_shift + tmean_c);
    put(M_THICK_D_MAX, tmax_);
    put(M_THICK_D_MIN, tmin_);
    put(M_THICK_D_STD, sqrtf(fmaxf(r21 / (float)NTN - tmean_c * tmean_c, 0.f)));
  } else if (q == 15) {
    const float nmean_c = r22 / (float)S;
    put(M_THIN_D_MEAN, n_shift + nmean_c);
    put(M_THIN_D_MAX, nmax_);
    put(M_THIN_D_MIN, nmin_);
    put(M_THIN_D_STD, sqrtf(fmaxf(r23 / (float)S - nmean_c * nmean_c, 0.f)));
  } else if (q == 16) {
    const float fth = (float)T.n_thick;
    put(M_THICK_E_AVG, en_new / fth);
    put(M_THICK_E_DELTA, en_delta / fth);
    put(M_TITIN_E_AVG, ten_new / fth);
    put(M_TITIN_E_DELTA, ten_delta / fth);
  } else if (q == 17) {
    const float work = force * (r24 / (float)NTN);
    put(M_WORK_THICK, work);
    put(M_WORK_THICK_MEAN, work / (float)NTN);
    put(M_WORK_PER_ATP, r25 > 0.01f ? work / r25 : 0.0f);
  }
  // the next step's pre-step snapshot: every read of this one (the partial
  // sums above) ended at the barrier, and the step's closing barrier orders
  // these copies before the next kinetics changes the state
  for (int i = tid; i < NTN; i += NT) m.s.old_thick[i] = m.s.x[i];
  for (int i = tid; i < X; i += NT) {
    m.s.old_xbs[i] = m.s.xb_state[i];
    m.s.old_key[i] = m.s.xb_key[i];
  }
  MF_MT(5);
#undef MF_MT
}

// ---------------------------------------------------------------------------
// one CTA = one condition, steps [t_begin, t_end)
// ---------------------------------------------------------------------------
#ifdef MF_PHASE_TIMING
// Diagnostic build only: thread 0 accumulates clock64() per phase and writes
// the totals over the x_trace test-hook buffer at the end of the launch.
#define MF_PH(k)                                  \
  do {                                            \
    __syncthreads();                              \
    if (m.tid == 0) {                             \
      const long long now_ = clock64();           \
      ph_sh[ph_cur] += (double)(now_ - ph_t0);    \
      ph_t0 = now_;                               \
      ph_cur = (k);                               \
    }                                             \
  } while (0)
#else
#define MF_PH(k) do { } while (0)
#endif

template <int NT, bool PR, bool DY>
__device__ void run_condition(const StepArgs& A, int ci) {
#ifdef MF_PHASE_TIMING
  // totals in shared memory: a runtime-indexed local array would add a
  // local-memory round trip to every marker
  __shared__ double ph_sh[28];
  if (threadIdx.x < 28) ph_sh[threadIdx.x] = 0.0;
  long long ph_t0 = clock64();
  int ph_cur = 0;
#endif
  extern __shared__ __align__(16) char smem_raw[];
  __shared__ CondDesc sh_cd;
  __shared__ TopoDev sh_T;
  __shared__ Smem sh_s;
  __shared__ CoefLayout sh_cl;
  __shared__ SlotLayout sh_L;
  if (threadIdx.x == 0) {
    sh_cd = A.cond[ci];
    sh_T = *sh_cd.topo;
    sh_cl = coef_layout(sh_T);
    sh_L = slot_layout(sh_T.n_dof, sh_T.total_xbs, sh_T.n_sites_total, sh_T.n_bins, sh_cl.total, A.pop.kx(),
                       A.pop.kt());
  }
  __syncthreads();
  const CondDesc& cd = sh_cd;
  const TopoDev& T = sh_T;
  Sim<NT, PR, DY> m(T, A, sh_s, sh_cl, sh_L);
#ifdef MF_PHASE_TIMING
  m.sub_acc = ph_sh + 12;
#endif
  m.tid = threadIdx.x;
  m.lane = m.tid & 31;
  m.warp = m.tid >> 5;
  m.b = cd.index;
  m.ws = cd.ws;
  m.set_dyn(DY);
  m.part = (A.flags & FLAG_ORIG_PRNG) == 0;
  m.status = 0;
  m.Tstride = cd.T;
  const int layout = (A.flags & FLAG_VEC_GLOBAL) ? LAYOUT_GLOBAL : ((A.flags & FLAG_REGS) ? LAYOUT_REGS : LAYOUT_SMEM);
  if (m.tid == 0) {
    carve(m, smem_raw, layout);
    m.s.tab.dtm = cd.dt;
  }
  __syncthreads();
  m.lazy_tab = DY && m.lazy_tables_fit();
  // the host sets FLAG_REGS exactly when regcg_fits, n_cg > 0 and the
  // precise mode hold (the register layout has no room for the other CG)
  m.regcg = PR && layout == LAYOUT_REGS;
  const int b = m.b;
  const int N = T.n_dof, X = T.total_xbs, S = T.n_sites_total, NTN = T.n_thick_nodes;
  // Workspace arrays of this condition, formed where they are used (launch
  // start and end) so that none of the pointers stays live across the step
  // loop.
#define MF_WS(type, field) reinterpret_cast<type*>(m.ws + m.L.field)

  for (int i = m.tid; i < kNParams; i += NT) m.s.P[i] = cd.params[i];
  if (A.pop.active()) {
    // population rows and fractions; labels clamped to [0, K)
    const int K = A.pop.K;
    for (int i = m.tid; i < K * kNParams; i += NT) m.s.Pk[i] = cd.pop_params[i];
    for (int i = m.tid; i < K; i += NT) m.s.fk[i] = cd.pop_frac ? cd.pop_frac[i] : 0.f;
    if (A.pop.kx() > 1)
      for (int i = m.tid; i < X; i += NT) m.s.xlab[i] = (int8_t)min(max((int)cd.xb_label[i], 0), K - 1);
    if (A.pop.kt() > 1)
      for (int g = m.tid; g < S; g += NT) m.s.tlab[g] = (int8_t)min(max((int)cd.tm_label[g], 0), K - 1);
  }
  m.Kl = cd.K_lat;
  m.nu_c = cd.nu;
  m.dtm = cd.dt;
  const float* zt = cd.z;
  const float* pt = cd.pCa;
  const float* lt = cd.ls;
  const int ds = cd.drv_const ? 0 : 1;  // driver index step per timestep
  const int n_steps = cd.n_steps;
  const int t0 = cd.t0;
  const int t1 = cd.t1 < n_steps ? cd.t1 : n_steps;
  if (t0 >= t1 && t0 > 0) return;
  __syncthreads();

  __shared__ uint32_t key_s[2];
  __shared__ float ls_s;
  // (pCa, d) of the sampling and absorbing tables in the workspace and the
  // initial z: read from shared memory every step, persisted at launch end
  __shared__ double tab_key[5];
  __shared__ int samp_est;  // key count of the last sampling build (dynamic spacing; 0: none yet)
  if (t0 == 0) {
    // ---- realize_state + initial equilibrium with the constants (A1) ----
    m.zref = (double)zt[0];
    for (int i = m.tid; i < N; i += NT) {
      if (i < NTN) m.s.x[i] = m.precise ? 0.f : T.crown_off[i];
      else m.s.x[i] = m.precise ? 0.f : zt[0] - T.bind_off[i - NTN];
    }
    for (int i = m.tid; i < X; i += NT) {
      m.s.xb_state[i] = 0;
      m.s.xb_bound[i] = -1;
    }
    for (int g = m.tid; g < S; g += NT) {
      m.s.tm[g] = 0;
      m.s.thin_bound[g] = -1;
    }
    m.build_precond_coef(MF_WS(float, coef));
    __syncthreads();
    __threadfence_block();
    for (int i = m.tid; i < m.cl.total; i += NT) m.s.coef[i] = MF_WS(float, coef)[i];
    __syncthreads();
    // the initial equilibrium itself runs as step -1 of the loop below, so
    // that the nearest-site search and the solver have one call site each
  } else {
    // ---- resume a condition from its resident workspace ----
    m.zref = MF_WS(double, misc)[MS_ZREF];
    for (int i = m.tid; i < N; i += NT) m.s.x[i] = MF_WS(float, x)[i];
    for (int i = m.tid; i < X; i += NT) {
      m.s.xb_state[i] = MF_WS(int8_t, xb_state)[i];
      m.s.xb_bound[i] = MF_WS(int16_t, xb_bound)[i];
      m.s.xb_near[i] = MF_WS(int16_t, xb_near)[i];
      m.s.xb_ax[i] = MF_WS(float, xb_ax)[i];
      m.s.xb_key[i] = MF_WS(int16_t, xb_key)[i];
    }
    for (int g = m.tid; g < S; g += NT) {
      m.s.tm[g] = MF_WS(int8_t, tm)[g];
      m.s.thin_bound[g] = MF_WS(int16_t, thin_bound)[g];
    }
    for (int i = m.tid; i < m.cl.total; i += NT) m.s.coef[i] = MF_WS(float, coef)[i];
    for (int i = m.tid; i < A.pop.kt() * 27 * 16; i += NT) m.s.cum_tm[i] = MF_WS(float, cum_tm)[i];
    for (int i = m.tid; i < A.pop.kx() * 6 * T.n_bins; i += NT) m.s.pabs[i] = MF_WS(float, pabs)[i];
    if (m.tid == 0) {
      const uint32_t* kk = reinterpret_cast<const uint32_t*>(MF_WS(double, misc) + MS_KEY);
      key_s[0] = kk[0];
      key_s[1] = kk[1];
      ls_s = (float)MF_WS(double, misc)[MS_CUR_LS];
      m.status = (int)MF_WS(double, misc)[MS_STATUS];
      tab_key[0] = MF_WS(double, misc)[MS_TAB_PCA];
      tab_key[1] = MF_WS(double, misc)[MS_TAB_D];
      tab_key[2] = MF_WS(double, misc)[MS_ABS_PCA];
      tab_key[3] = MF_WS(double, misc)[MS_ABS_D];
      tab_key[4] = MF_WS(double, misc)[MS_L0];
    }
    __syncthreads();
  }

  // Sub-keys of step t in slot t & 1.  The keys of step t + 1 are derived
  // during step t by the CTA's last thread, which has the fewest sites in
  // the tropomyosin update (keys_ready), so the serial Threefry chain leaves
  // the start of the step; otherwise thread 0 derives them there.
  __shared__ uint32_t sub_thin[2][2], sub_thick[2][2];
  __shared__ int keys_ready;
  if (m.tid == 0) {
    keys_ready = 0;
    samp_est = 0;  // no merged build before a sampling build has counted the keys
  }
  // Drivers (z, pCa, ls) of step t in drv[t & 1].  Thread 0 copies those of
  // step t + 1 with cp.async during step t: their latency overlaps a whole
  // step, and no register holds them (or the driver pointers) across the
  // step's phases, whose peak register demand is the solver's.
  __shared__ float drv[2][3];
  __shared__ float prev_z_s;
  if (m.tid == 0) {
    if (t0 < t1) {
      drv[t0 & 1][0] = zt[t0 * ds];
      drv[t0 & 1][1] = pt[t0 * ds];
      drv[t0 & 1][2] = lt[t0 * ds];
    }
    prev_z_s = t0 > 0 ? zt[(t0 - 1) * ds] : 0.0f;
  }
  __syncthreads();
  // t = -1: the initial equilibrium with the constants (A1): nearest sites
  // at the constant spacing, table rows of the initial geometry, one solve
  // at the constant z_line with the spacing held fixed.
  for (int t = t0 == 0 ? -1 : t0; t < t1; ++t) {
    const bool init = t < 0;
    float zl, pCa = 0.0f, ls_t = 0.0f, cur_ls = 0.0f, d_kin;
    if (init) {
      zl = m.s.P[Z_LINE];
      d_kin = m.s.P[LATTICE_SPACING];
    } else {
      zl = drv[t & 1][0];
      pCa = drv[t & 1][1];
      ls_t = drv[t & 1][2];
      const float dz = t > 0 ? zl - prev_z_s : 0.0f;
      if (m.tid == 0 && t + 1 < t1) {
        float* nx = drv[(t + 1) & 1];
        cp_async4(nx + 0, cd.z + (t + 1) * ds);
        cp_async4(nx + 1, cd.pCa + (t + 1) * ds);
        cp_async4(nx + 2, cd.ls + (t + 1) * ds);
      }
      // 1. rigid shift of the thin filaments
      if (!m.precise) {
        for (int i = NTN + m.tid; i < N; i += NT) m.s.x[i] = m.s.x[i] + dz;
      } else {
        m.zref = (double)zl;
      }
      cur_ls = ls_s;
      if (m.dyn) {
        d_kin = cur_ls;
        const float l0 = (float)tab_key[4];
        m.d_ref = ls_t * powf(l0 / zl, m.nu_c);
      } else {
        d_kin = ls_t;
      }
      MF_PH(1);
      // probability tables for (pCa, d_kin); with a dynamic spacing the
      // crossbridge rows are built after the tropomyosin update instead
      if (DY && m.lazy_tab) {
        // tab_key[1]: the spacing at which every sampling row was built
        // (together with the absorbing rows of the step before), NaN when
        // the rows are of mixed keys
        if ((double)pCa != tab_key[0]) {
          __syncthreads();
          m.build_tm_tables(pCa);
          __syncthreads();
          if (m.tid == 0) {
            tab_key[0] = pCa;
            tab_key[1] = NAN;
          }
          __syncthreads();
        }
      } else if (!((double)pCa == tab_key[0] && (double)d_kin == tab_key[1])) {
        // with a fixed spacing the metrics' absorbing table has the same
        // (pCa, spacing) key: both are built in one pass over the CTA's
        // threads (fewer partly filled rounds of one matrix per thread)
        const bool abs_too = !DY && !((double)pCa == tab_key[2] && (double)d_kin == tab_key[3]);
        __syncthreads();
        m.build_tables(pCa, d_kin, true, abs_too);
        __syncthreads();
        if (m.tid == 0) {
          tab_key[0] = pCa;
          tab_key[1] = d_kin;
          if (abs_too) { tab_key[2] = pCa; tab_key[3] = d_kin; }
        }
        __threadfence_block();
        __syncthreads();
      }
      MF_PH(2);
      // old_state snapshot for the metrics (metrics_fn.py reads the pre-step
      // geometry): taken here at the first step of a launch, afterwards by the
      // previous step's metrics epilogue
      const bool first = t == (t0 > 0 ? t0 : 0);
      if (first) {
        for (int i = m.tid; i < NTN; i += NT) m.s.old_thick[i] = m.s.x[i];
        for (int i = m.tid; i < X; i += NT) {
          m.s.old_xbs[i] = m.s.xb_state[i];
          m.s.old_key[i] = m.s.xb_key[i];
        }
      }
      if (m.tid == 0) {
        if (!keys_ready) {
          uint32_t kn[2];
          step_keys(m.part, key_s[0], key_s[1], sub_thin[t & 1], sub_thick[t & 1], kn);
          key_s[0] = kn[0];
          key_s[1] = kn[1];
        }
        keys_ready = 0;
      }
      // the shifted thin positions (float32 mode) must be complete before the
      // nearest-site staging reads them; the keys are read after its barriers
      if (first || !m.precise) __syncthreads();
      MF_PH(3);
    }
    // 2-4. kinetics.  No barrier after the nearest-site search: the
    // tropomyosin sampling reads none of its outputs, the initial key loop
    // reads only its own heads' offsets, and thin_step's first barrier
    // precedes the bid arrays it writes over the staged face positions.
    m.nearest(d_kin);
    MF_PH(4);
    if (init) {
      // table rows of the initial geometry (every site starts in state 0: block 0)
      for (int i = m.tid; i < X; i += NT) m.s.xb_key[i] = (int16_t)(m.pop_key(i) + m.bin_of(m.s.xb_ax[i]));
    } else {
      const size_t inj_t = ((size_t)b * A.T + t) * (size_t)S;
      const size_t inj_x = ((size_t)b * A.T + t) * (size_t)X;
      m.thin_step(sub_thin[t & 1], inj_t, [&]() {
        if (m.tid == NT - 1 && t + 1 < t1) {
          uint32_t kn[2];
          step_keys(m.part, key_s[0], key_s[1], sub_thin[(t + 1) & 1], sub_thick[(t + 1) & 1], kn);
          key_s[0] = kn[0];
          key_s[1] = kn[1];
          keys_ready = 1;
        }
      });
      if (DY && m.lazy_tab && !((double)d_kin == tab_key[1])) {
        const int nk = m.build_needed_tables(pCa, d_kin, false);
        if (m.tid == 0) {
          samp_est = nk;
          tab_key[1] = NAN;
#ifdef MF_PHASE_TIMING
          m.sub_acc[5] += 1.0;  // sampling builds
          m.sub_acc[7] += nk;   // their keys
#endif
        }
      }
      MF_PH(5);
      m.thick_step(sub_thick[t & 1], inj_x);
      MF_PH(6);
    }
    // 5. mechanics
    double resid;
    int iters;
    const bool dyn_save = m.dyn;
    m.set_dyn(dyn_save && !init);
    float d = init ? d_kin : (m.dyn ? cur_ls : ls_t);
    m.build_bound_list();
    MF_PH(7);
    m.solve(zl, d, resid, iters, m.dyn);
    MF_PH(8);
    m.set_dyn(dyn_save);
    if (init) {
      if (m.tid == 0) {
        key_s[0] = cd.key[0];
        key_s[1] = cd.key[1];
        ls_s = cd.ls[0];
        tab_key[0] = NAN;
        tab_key[1] = NAN;
        tab_key[2] = NAN;
        tab_key[3] = NAN;
        tab_key[4] = (double)cd.z[0];
      }
      __syncthreads();
      continue;
    }
    // the step's drivers again from shared memory: their registers are free
    // during the solve
    zl = drv[t & 1][0];
    pCa = drv[t & 1][1];
    ls_t = drv[t & 1][2];
    const float new_ls = m.dyn ? d : ls_t;
    if (m.tid == 0) ls_s = new_ls;
    // absorbing table for the metrics at (pCa, new_ls)
    if (DY && m.lazy_tab) {
      // with pCa unchanged at step t + 1 its sampling rows may be built here
      if (m.tid == 0 && t + 1 < t1) cp_async_wait_all();  // step t + 1's drivers
      __syncthreads();
      const bool same_next = t + 1 < t1 && drv[(t + 1) & 1][1] == pCa;
      const int all = m.build_needed_tables(pCa, new_ls, true, same_next, samp_est);
      if (all && m.tid == 0) {
        tab_key[1] = new_ls;
#ifdef MF_PHASE_TIMING
        m.sub_acc[6] += 1.0;  // absorbing builds that built every sampling row too
#endif
      }
    } else if (!((double)pCa == tab_key[2] && (double)new_ls == tab_key[3])) {
      __syncthreads();
      m.build_tables(pCa, new_ls, false, true);
      __syncthreads();
      if (m.tid == 0) { tab_key[2] = pCa; tab_key[3] = new_ls; }
      __threadfence_block();
    }
    __syncthreads();
    MF_PH(9);
    // 6. force + metrics
    metrics(m, t, zl, pCa, new_ls, resid, iters, cd.metrics);
    if (resid > (double)A.resid_warn) m.status |= 2;
    MF_PH(10);
    // optional traces
    if (A.x_trace) {
      float* xt = A.x_trace + ((size_t)b * A.T + t) * A.max_dof;
      for (int i = m.tid; i < N; i += NT) {
        float v = m.s.x[i];
        if (m.precise) {
          v = i < NTN ? (float)((double)T.crown_off[i] + (double)v)
                      : (float)((m.zref - (double)T.bind_off[i - NTN]) + (double)v);
        }
        xt[i] = v;
      }
    }
    if (A.st_trace) {
      int8_t* st = A.st_trace + ((size_t)b * A.T + t) * (A.max_xbs + A.max_sites);
      int* bt = A.bd_trace + ((size_t)b * A.T + t) * (A.max_xbs + A.max_sites);
      for (int i = m.tid; i < X; i += NT) { st[i] = m.s.xb_state[i]; bt[i] = m.s.xb_bound[i]; }
      for (int g = m.tid; g < S; g += NT) { st[A.max_xbs + g] = m.s.tm[g]; bt[A.max_xbs + g] = m.s.thin_bound[g]; }
    }
    if (m.tid == 0) {
      prev_z_s = zl;
      cp_async_wait_all();  // step t + 1's drivers, published by the barrier below
    }
    __syncthreads();
  }
  MF_PH(11);
#ifdef MF_PHASE_TIMING
  if (m.tid == 0 && A.x_trace) {
    float* o = A.x_trace + (size_t)b * A.T * A.max_dof;
    for (int k = 0; k < 28; ++k) o[k] = (float)ph_sh[k];
  }
#endif
  // ---- write back resident state ----
  for (int i = m.tid; i < N; i += NT) MF_WS(float, x)[i] = m.s.x[i];
  for (int i = m.tid; i < X; i += NT) {
    MF_WS(int8_t, xb_state)[i] = m.s.xb_state[i];
    MF_WS(int16_t, xb_bound)[i] = m.s.xb_bound[i];
    MF_WS(int16_t, xb_near)[i] = m.s.xb_near[i];
    MF_WS(float, xb_ax)[i] = m.s.xb_ax[i];
    MF_WS(int16_t, xb_key)[i] = m.s.xb_key[i];
  }
  for (int g = m.tid; g < S; g += NT) {
    MF_WS(int8_t, tm)[g] = m.s.tm[g];
    MF_WS(int16_t, thin_bound)[g] = m.s.thin_bound[g];
  }
  for (int i = m.tid; i < A.pop.kt() * 27 * 16; i += NT) MF_WS(float, cum_tm)[i] = m.s.cum_tm[i];
  for (int i = m.tid; i < A.pop.kx() * 6 * T.n_bins; i += NT) MF_WS(float, pabs)[i] = m.s.pabs[i];
  // block-wide OR of the status bits (__syncthreads_or returns 0 or 1, not
  // the OR of its operands, so each bit is reduced on its own)
  int st_all = 0;
  for (int bit = 1; bit <= 8; bit <<= 1) st_all |= __syncthreads_or(m.status & bit) ? bit : 0;
  if (m.tid == 0) {
    uint32_t* kk = reinterpret_cast<uint32_t*>(MF_WS(double, misc) + MS_KEY);
    kk[0] = key_s[0];
    kk[1] = key_s[1];
    MF_WS(double, misc)[MS_CUR_LS] = ls_s;
    MF_WS(double, misc)[MS_ZREF] = m.zref;
    MF_WS(double, misc)[MS_STATUS] = (double)(m.status | st_all);
    MF_WS(double, misc)[MS_TAB_PCA] = tab_key[0];
    MF_WS(double, misc)[MS_TAB_D] = tab_key[1];
    MF_WS(double, misc)[MS_ABS_PCA] = tab_key[2];
    MF_WS(double, misc)[MS_ABS_D] = tab_key[3];
    MF_WS(double, misc)[MS_L0] = tab_key[4];
    if (cd.status) *cd.status = m.status | st_all;
    if (cd.key_out) { cd.key_out[0] = key_s[0]; cd.key_out[1] = key_s[1]; }
  }
}
#undef MF_WS

// Register cap of 128 per thread (80 at 384 threads, 64 at 1024) so that
// several conditions share an SM; the table builder's 6x6 temporaries spill
// instead.  min_ctas: resident CTAs per SM the register budget is sized for.
constexpr int min_ctas(int nt) { return nt == 384 ? 2 : ((65536 / (nt * 128)) > 0 ? 65536 / (nt * 128) : 1); }

// PR: precise (mixed) mode, a compile-time choice so that each kernel holds
// only its own solver.  DY: dynamic lattice spacing; without it the radial
// unknown and its recurrences are compiled out of the solver, which frees
// the registers they hold through the CG loop.
template <int NT, bool PR, bool DY>
__global__ void __launch_bounds__(NT, min_ctas(NT))
    step_kernel(StepArgs A, int cond_base) {
  run_condition<NT, PR, DY>(A, cond_base + blockIdx.x);
}

}  // namespace mf
