// One step of caller-owned states: the public kinetics / equilibrium split.
//
// The fused kernel (mf_kernel.cuh) keeps a condition's state on chip for a
// whole run.  The reference also exposes the halves of a timestep as
// functions of an explicit State (timestep.py:65-199: kinetics_step,
// timestep; kernels/geometry.py:186-262: update_nearest_neighbors;
// kernels/solver.py:663-771: solve_equilibrium), which coupled
// multi-sarcomere solvers call between their own steps.  state_kernel runs
// any of those phases on B states held by the caller in the reference's
// State layout (core/state.py:69-113), one CTA per state, with the fused
// kernel's own phase code (Sim): it loads a state into shared memory, runs
// the phases and stores it back.  Arithmetic is the reference's float32
// (absolute positions).
#pragma once
#include "mf_kernel.cuh"

namespace mf {

// phase bits of a call
constexpr int PHASE_NEAREST = 1, PHASE_TRANSITIONS = 2, PHASE_EQUILIBRIUM = 4;

// The caller's state arrays ([B, ...] each, device) and per-state inputs.
struct StateIO {
  const TopoDev* topo;
  char* ws;             // workspace, ws_stride bytes per state (tables, large-lattice vectors)
  size_t ws_stride;
  float* thick_axial;   // [B, n_thick * n_crowns]
  int8_t* xb_states;    // [B, X]
  int32_t* xb_bound;    // [B, X]
  int32_t* xb_nearest;  // [B, X]
  float* xb_dist;       // [B, X, 2]
  float* thin_axial;    // [B, S]
  int8_t* tm_states;    // [B, S]
  int32_t* thin_bound;  // [B, S]
  uint32_t* keys;       // [B, 2] in / out
  const float* params;  // [B, 44]
  const float* pCa;     // [B] drivers; NaN = the constant (state.py:331-343)
  const float* z;
  const float* ls;
  const float* K_lat;   // [B] (dynamic spacing)
  const float* d_ref;   // [B] (dynamic spacing)
  float* resid_out;     // [B] or NULL
  float* ls_out;        // [B] or NULL
  int32_t* iters_out;   // [B] or NULL
  int32_t* status_out;  // [B] or NULL
  // subpopulations: [B, K, 44], [B, K], [B, label_stride] x 2
  const float* pop_params;
  const float* pop_frac;
  const int8_t* xb_label;
  const int8_t* tm_label;
  int label_stride;
  int phases;
  float dt;
};

template <int NT, bool DY>
__device__ void run_state(const StepArgs& A, const StateIO& io, int b) {
  extern __shared__ __align__(16) char smem_raw[];
  __shared__ TopoDev sh_T;
  __shared__ Smem sh_s;
  __shared__ CoefLayout sh_cl;
  __shared__ SlotLayout sh_L;
  __shared__ uint32_t key_s[2], sub_thin[2], sub_thick[2];
  __shared__ float drv[3];
  if (threadIdx.x == 0) {
    sh_T = *io.topo;
    sh_cl = coef_layout(sh_T);
    sh_L = slot_layout(sh_T.n_dof, sh_T.total_xbs, sh_T.n_sites_total, sh_T.n_bins, sh_cl.total, A.pop.kx(),
                       A.pop.kt());
  }
  __syncthreads();
  const TopoDev& T = sh_T;
  Sim<NT, false, DY> m(T, A, sh_s, sh_cl, sh_L);
  m.tid = threadIdx.x;
  m.lane = m.tid & 31;
  m.warp = m.tid >> 5;
  m.b = b;
  m.ws = io.ws + (size_t)b * io.ws_stride;
  m.part = (A.flags & FLAG_ORIG_PRNG) == 0;
  m.status = 0;
  m.Tstride = 1;
  m.zref = 0.0;
  m.regcg = false;
  m.lazy_tab = false;
  const int layout = (A.flags & FLAG_VEC_GLOBAL) ? LAYOUT_GLOBAL : LAYOUT_SMEM;
  if (m.tid == 0) {
    carve(m, smem_raw, layout);
    m.s.tab.dtm = io.dt;
  }
  __syncthreads();
  const int N = T.n_dof, X = T.total_xbs, S = T.n_sites_total, NTN = T.n_thick_nodes;
  const float* prow = io.params + (size_t)b * kNParams;
  for (int i = m.tid; i < kNParams; i += NT) m.s.P[i] = prow[i];
  if (A.pop.active()) {
    const int K = A.pop.K;
    const float* pk = io.pop_params + (size_t)b * K * kNParams;
    for (int i = m.tid; i < K * kNParams; i += NT) m.s.Pk[i] = pk[i];
    for (int i = m.tid; i < K; i += NT) m.s.fk[i] = io.pop_frac ? io.pop_frac[(size_t)b * K + i] : 0.f;
    if (A.pop.kx() > 1)
      for (int i = m.tid; i < X; i += NT)
        m.s.xlab[i] = (int8_t)min(max((int)io.xb_label[(size_t)b * io.label_stride + i], 0), K - 1);
    if (A.pop.kt() > 1)
      for (int g = m.tid; g < S; g += NT)
        m.s.tlab[g] = (int8_t)min(max((int)io.tm_label[(size_t)b * io.label_stride + g], 0), K - 1);
  }
  // the caller's state
  for (int i = m.tid; i < N; i += NT)
    m.s.x[i] = i < NTN ? io.thick_axial[(size_t)b * NTN + i] : io.thin_axial[(size_t)b * S + (i - NTN)];
  for (int i = m.tid; i < X; i += NT) {
    const size_t o = (size_t)b * X + i;
    m.s.xb_state[i] = io.xb_states[o];
    m.s.xb_bound[i] = (int16_t)io.xb_bound[o];
    m.s.xb_near[i] = (int16_t)io.xb_nearest[o];
    m.s.xb_ax[i] = io.xb_dist[2 * o];
  }
  for (int g = m.tid; g < S; g += NT) {
    const size_t o = (size_t)b * S + g;
    m.s.tm[g] = io.tm_states[o];
    m.s.thin_bound[g] = (int16_t)io.thin_bound[o];
  }
  if (m.tid == 0) {
    // drivers resolved against the constants (resolve_value: NaN -> constant)
    const float pc = io.pCa ? io.pCa[b] : NAN, zz = io.z ? io.z[b] : NAN, ll = io.ls ? io.ls[b] : NAN;
    drv[0] = pc == pc ? pc : prow[PCA];
    drv[1] = zz == zz ? zz : prow[Z_LINE];
    drv[2] = ll == ll ? ll : prow[LATTICE_SPACING];
    key_s[0] = io.keys[2 * b];
    key_s[1] = io.keys[2 * b + 1];
  }
  m.Kl = DY ? io.K_lat[b] : 0.f;
  m.d_ref = DY ? io.d_ref[b] : 0.f;
  m.nu_c = 0.f;
  m.dtm = io.dt;
  m.set_dyn(DY);
  if (io.phases & PHASE_EQUILIBRIUM) {
    m.build_precond_coef(reinterpret_cast<float*>(m.ws + m.L.coef));
    __syncthreads();
    __threadfence_block();
    for (int i = m.tid; i < m.cl.total; i += NT) m.s.coef[i] = reinterpret_cast<float*>(m.ws + m.L.coef)[i];
  }
  __syncthreads();
  const float pCa = drv[0], zl = drv[1], ls = drv[2];
  if (io.phases & PHASE_TRANSITIONS) {
    // this step's sub-keys (timestep.py:120,125) and the sampling tables
    if (m.tid == 0) {
      uint32_t kn[2];
      step_keys(m.part, key_s[0], key_s[1], sub_thin, sub_thick, kn);
      key_s[0] = kn[0];
      key_s[1] = kn[1];
    }
    m.build_tables(pCa, ls, true, false);
    __syncthreads();
    __threadfence_block();
  }
  if (io.phases & PHASE_NEAREST) {
    m.nearest(ls);
    __syncthreads();
  }
  if (io.phases & PHASE_TRANSITIONS) {
    m.thin_step(sub_thin, (size_t)b * S, []() {});
    m.thick_step(sub_thick, (size_t)b * X);
  }
  if (io.phases & PHASE_EQUILIBRIUM) {
    double resid;
    int iters;
    float d = ls;
    m.build_bound_list();
    m.solve(zl, d, resid, iters, m.dyn);
    __syncthreads();
    if (m.tid == 0) {
      if (io.resid_out) io.resid_out[b] = (float)resid;
      if (io.ls_out) io.ls_out[b] = d;
      if (io.iters_out) io.iters_out[b] = iters;
    }
  }
  __syncthreads();
  // the state back to the caller
  if (io.phases & PHASE_EQUILIBRIUM)
    for (int i = m.tid; i < N; i += NT) {
      if (i < NTN) io.thick_axial[(size_t)b * NTN + i] = m.s.x[i];
      else io.thin_axial[(size_t)b * S + (i - NTN)] = m.s.x[i];
    }
  for (int i = m.tid; i < X; i += NT) {
    const size_t o = (size_t)b * X + i;
    io.xb_states[o] = m.s.xb_state[i];
    io.xb_bound[o] = m.s.xb_bound[i];
    if (io.phases & PHASE_NEAREST) {
      io.xb_nearest[o] = m.s.xb_near[i];
      io.xb_dist[2 * o] = m.s.xb_ax[i];
      io.xb_dist[2 * o + 1] = ls;
    }
  }
  for (int g = m.tid; g < S; g += NT) {
    const size_t o = (size_t)b * S + g;
    io.tm_states[o] = m.s.tm[g];
    io.thin_bound[o] = m.s.thin_bound[g];
  }
  int st_all = 0;
  for (int bit = 1; bit <= 8; bit <<= 1) st_all |= __syncthreads_or(m.status & bit) ? bit : 0;
  if (m.tid == 0) {
    io.keys[2 * b] = key_s[0];
    io.keys[2 * b + 1] = key_s[1];
    if (io.status_out) io.status_out[b] = st_all;
  }
}

template <int NT, bool DY>
__global__ void __launch_bounds__(NT, min_ctas(NT)) state_kernel(StepArgs A, StateIO io) {
  run_state<NT, DY>(A, io, blockIdx.x);
}

}  // namespace mf
