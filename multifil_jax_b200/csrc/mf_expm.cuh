// Rate matrices and the binned Pade(6,6) matrix exponential.
//
// Restates kernels/transitions.py:99-190 (expm_pade6_batch),
// :434-513 (27 tropomyosin generators), :632-804 (crossbridge generator) with
// the rate laws of kernels/rate_functions.py:165-753.  The tables depend only
// on (params, pCa, lattice spacing, dt), so they are built once per condition
// whenever those inputs are constant and once per step otherwise.
//
// One matrix is owned by a group of 8 consecutive lanes: lane r of the group
// holds row r (r < N; the other lanes of the group compute on a copy of the
// last row and store nothing).  Products, the pivot search, the row
// exchanges and the back substitution move rows between the group's lanes
// with width-8 shuffles, so a lane holds a few rows of registers instead of
// whole matrices, and four matrices of a warp advance together.  The
// squaring phase optionally runs in float64.
#pragma once
#include "mf_common.cuh"

namespace mf {

__constant__ float kPade6B[7] = {1.0f, 1.0f / 2.0f, 1.0f / 9.0f, 1.0f / 72.0f, 1.0f / 1008.0f,
                                 1.0f / 30240.0f, 1.0f / 1209600.0f};

constexpr int kGroup = 8;  // lanes per matrix

// Row r of C = A B from row r of A (a) and the rows of B held by the group's
// lanes (b): C[r][k] = A[r][0] B[0][k] + ... in increasing j, one fused
// multiply-add per further term.
template <int N, class F>
__device__ __forceinline__ void mm_row(unsigned gmask, const F (&a)[N], const F (&b)[N], F (&c)[N]) {
  F bj[N];
#pragma unroll
  for (int k = 0; k < N; ++k) bj[k] = __shfl_sync(gmask, b[k], 0, kGroup);
#pragma unroll
  for (int k = 0; k < N; ++k) c[k] = a[0] * bj[k];
#pragma unroll
  for (int j = 1; j < N; ++j) {
#pragma unroll
    for (int k = 0; k < N; ++k) bj[k] = __shfl_sync(gmask, b[k], j, kGroup);
#pragma unroll
    for (int k = 0; k < N; ++k) c[k] = fma(a[j], bj[k], c[k]);
  }
}

// exp(A) of the group's matrix, row r in a[] (in place).  Returns the
// squaring count s (2^s >= ||A||_inf / 0.5).  sq64_from: the squarings run
// in float64 when s >= sq64_from (a large value keeps them in float32).
// Every lane of the 8-lane group takes part (gmask names the group).
template <int N>
__device__ int expm_rows(unsigned gmask, int r, float (&a)[N], int sq64_from) {
  const bool own = r < N;
  // infinity norm: the largest absolute row sum (NaN-propagating, as jnp.max)
  float rs = fabsf(a[0]);
#pragma unroll
  for (int j = 1; j < N; ++j) rs += fabsf(a[j]);
  float nrm = own ? rs : 0.f;
#pragma unroll
  for (int o = 1; o < kGroup; o <<= 1) nrm = fmax_nan(nrm, __shfl_xor_sync(gmask, nrm, o, kGroup));
  int s = (int)ceilf(log2f(nrm / 0.5f + 1e-10f));
  s = s < 0 ? 0 : s;
  const float inv = 1.0f / exp2f((float)s);  // exact power of two
#pragma unroll
  for (int j = 0; j < N; ++j) a[j] = a[j] * inv;
  // V = b0 I + b2 A2 + b4 A4 + b6 A6 ;  U = A (b1 I + b3 A2 + b5 A4)
  float a2[N], a4[N], t[N], v[N], u[N];
  mm_row<N>(gmask, a, a, a2);
  mm_row<N>(gmask, a2, a2, a4);
  mm_row<N>(gmask, a4, a2, t);  // A6
#pragma unroll
  for (int j = 0; j < N; ++j) {
    const bool d = j == r;
    v[j] = (d ? kPade6B[0] : 0.f) + kPade6B[2] * a2[j] + kPade6B[4] * a4[j] + kPade6B[6] * t[j];
    t[j] = (d ? kPade6B[1] : 0.f) + kPade6B[3] * a2[j] + kPade6B[5] * a4[j];
  }
  mm_row<N>(gmask, a, t, u);
  // Solve (V - U) X = (V + U) by LU with partial pivoting (the first row of
  // largest magnitude in the column is the pivot).
  float L[N], R[N];
#pragma unroll
  for (int j = 0; j < N; ++j) {
    L[j] = v[j] - u[j];
    R[j] = v[j] + u[j];
  }
#pragma unroll
  for (int k = 0; k < N; ++k) {
    // pivot row: largest |L[i][k]| over rows i >= k, lowest index on ties
    float best = (own && r >= k) ? fabsf(L[k]) : -2.f;
    if (best != best) best = -1.f;
    int piv = own ? r : N;
#pragma unroll
    for (int o = 1; o < kGroup; o <<= 1) {
      const float ob = __shfl_xor_sync(gmask, best, o, kGroup);
      const int op = __shfl_xor_sync(gmask, piv, o, kGroup);
      if (ob > best || (ob == best && op < piv)) { best = ob; piv = op; }
    }
    if (piv >= N) piv = k;
    // exchange rows k and piv
    const int src = r == k ? piv : (r == piv ? k : r);
#pragma unroll
    for (int j = 0; j < N; ++j) {
      L[j] = __shfl_sync(gmask, L[j], src, kGroup);
      R[j] = __shfl_sync(gmask, R[j], src, kGroup);
    }
    // eliminate below the pivot with the pivot row
    float Lk[N], Rk[N];
#pragma unroll
    for (int j = 0; j < N; ++j) {
      Lk[j] = __shfl_sync(gmask, L[j], k, kGroup);
      Rk[j] = __shfl_sync(gmask, R[j], k, kGroup);
    }
    if (r > k) {
      const float l = L[k] / Lk[k];
#pragma unroll
      for (int j = k + 1; j < N; ++j) L[j] = L[j] - l * Lk[j];
#pragma unroll
      for (int j = 0; j < N; ++j) R[j] = R[j] - l * Rk[j];
    }
  }
  // back substitution, last row first: row i = (R[i] - sum_{m>i} L[i][m] X[m]) / L[i][i]
#pragma unroll
  for (int i = N - 1; i >= 0; --i) {
    if (r == i) {
#pragma unroll
      for (int j = 0; j < N; ++j) a[j] = R[j] / L[i];
    }
    float xi[N];
#pragma unroll
    for (int j = 0; j < N; ++j) xi[j] = __shfl_sync(gmask, a[j], i, kGroup);
    if (r < i) {
#pragma unroll
      for (int j = 0; j < N; ++j) R[j] = R[j] - L[i] * xi[j];
    }
  }
  if (!own) {  // keep the spare lanes' values finite and inert
#pragma unroll
    for (int j = 0; j < N; ++j) a[j] = 0.f;
  }
  // square s times (the reference caps the masked loop at 18 trips)
  const int nsq = s < 18 ? s : 18;
  if (nsq >= sq64_from) {
    // float64 squaring.  The Pade rows are first renormalised to unit sums:
    // rounding that moves a row sum off 1 is what 2^s squarings amplify (a
    // float64 squaring of an unrenormalised float32 result keeps ~5e-3 of
    // relative error at s = 16; renormalised, ~3e-6).
    double D[N], E[N];
    double sum = 0.0;
#pragma unroll
    for (int j = 0; j < N; ++j) sum += (double)a[j];
#pragma unroll
    for (int j = 0; j < N; ++j) D[j] = own ? (double)a[j] / sum : 0.0;
    for (int q = 0; q < nsq; ++q) {
      mm_row<N>(gmask, D, D, E);
#pragma unroll
      for (int j = 0; j < N; ++j) D[j] = E[j];
    }
    sum = 0.0;
#pragma unroll
    for (int j = 0; j < N; ++j) sum += D[j];
#pragma unroll
    for (int j = 0; j < N; ++j) a[j] = (float)(D[j] / sum);
  } else {
    float c[N];
    for (int q = 0; q < nsq; ++q) {
      mm_row<N>(gmask, a, a, c);
#pragma unroll
      for (int j = 0; j < N; ++j) a[j] = c[j];
    }
    float sum = a[0];
#pragma unroll
    for (int j = 1; j < N; ++j) sum += a[j];
#pragma unroll
    for (int j = 0; j < N; ++j) a[j] = a[j] / sum;
  }
#pragma unroll
  for (int j = 0; j < N; ++j)
    if (isnan(a[j])) a[j] = 1.0f / (float)N;
  return s;
}

// jnp.cumsum association for 4 and 6 entries (lax.associative_scan order).
__device__ __forceinline__ void cum4(const float* p, float* c) {
  const float s01 = p[0] + p[1];
  c[0] = p[0];
  c[1] = s01;
  c[2] = s01 + p[2];
  c[3] = s01 + (p[2] + p[3]);
}

__device__ __forceinline__ void cum6(const float* p, float* c) {
  const float s01 = p[0] + p[1];
  const float s0123 = s01 + (p[2] + p[3]);
  c[0] = p[0];
  c[1] = s01;
  c[2] = s01 + p[2];
  c[3] = s0123;
  c[4] = s0123 + p[4];
  c[5] = s0123 + (p[4] + p[5]);
}

// Row r (clamped to 3) of the tropomyosin generator of configuration
// cfg = 9*n2 + 3*n3 + n_closed (Ising coupling h; forward rates x e^{h/2},
// backward x e^{-h/2}).
static __device__ void tm_generator_row(const float* P, float pCa, int cfg, int r, float (&q)[4]) {
  const float ca = powf(10.0f, -pCa);
  const float n2 = (float)(cfg / 9), n3 = (float)((cfg / 3) % 3), nc = (float)(cfg % 3);
  const float JC = P[TM_J_C], JM = P[TM_J_M];
  const float h = JC * n2 + JM * n3 - 0.5f * (JC + JM) * nc;
  const float fwd = expf(0.5f * h), bwd = expf(-0.5f * h);
  const float k01 = P[TM_K_01] * ca * fwd;
  const float k12 = P[TM_K_12] * fwd;
  const float k23 = P[TM_K_23] * fwd;
  const float k30 = P[TM_K_30];
  const float k10 = (P[TM_K_01] / P[TM_KEQ_01]) * bwd;
  const float k21 = (P[TM_K_12] / P[TM_KEQ_12]) * bwd;
  const float k32 = (P[TM_K_23] / P[TM_KEQ_23]) * bwd;
  switch (r) {
    case 0: q[0] = -k01; q[1] = k01; q[2] = 0.f; q[3] = 0.f; break;
    case 1: q[0] = k10; q[1] = -(k10 + k12); q[2] = k12; q[3] = 0.f; break;
    case 2: q[0] = 0.f; q[1] = k21; q[2] = -(k21 + k23); q[3] = k23; break;
    default: q[0] = k30; q[1] = 0.f; q[2] = k32; q[3] = -(k30 + k32); break;
  }
}

// Row r (clamped to 5) of the crossbridge generator at axial offset x,
// spacing d, permissiveness perm.
static __device__ void xb_generator_row(const float* P, float pCa, float x, float d, float perm, int r,
                                        float (&q)[6]) {
  const float ca = powf(10.0f, -pCa);
  const float rr = sqrtf(x * x + d * d);
  const float th = atan2f(d, x);
  const float kt = 1.3810e-23f * (P[TEMP_CELSIUS] + 273.15f) * 1e21f;
  const float gw = rr - P[XB_G_REST_WEAK], cw = th - P[XB_C_REST_WEAK];
  const float gs = rr - P[XB_G_REST_STRONG], cs = th - P[XB_C_REST_STRONG];
  const float Ew = (0.5f * P[XB_G_K_WEAK] * (gw * gw) + 0.5f * P[XB_C_K_WEAK] * (cw * cw)) / kt;
  const float Es = (0.5f * P[XB_G_K_STRONG] * (gs * gs) + 0.5f * P[XB_C_K_STRONG] * (cs * cs)) / kt;
  const float Ediff = Ew - Es;
  const float U_drx = P[XB_U_DRX];
  const float U_loose = P[XB_U_LOOSE] + Ew;
  const float U_t1 = P[XB_U_TIGHT_1] + Es;
  const float U_t2 = P[XB_U_TIGHT_2] + Es;
  const float f_s = P[XB_G_K_STRONG] * gs + (1.0f / rr) * P[XB_C_K_STRONG] * cs;
  const float cap = 10000.0f;
#pragma unroll
  for (int j = 0; j < 6; ++j) q[j] = 0.f;
  float r01 = perm * P[XB_R01_COEFF] * expf(-Ew);
  if (isnan(r01)) r01 = 0.f;
  float r12 = P[XB_R12_COEFF] * expf(fmin_nan(Ediff, 30.0f) / 2.0f);
  if (isnan(r12)) r12 = 0.f;
  if (r == 0) {
    const float r04 = P[XB_R04], r05 = P[XB_R05];
    q[0] = -(r01 + r04 + r05); q[1] = r01; q[4] = r04; q[5] = r05;
  } else if (r == 1) {
    float r10 = fmin_nan(expf(logf(r01 + 0.005f) - (U_drx - U_loose)), cap);
    if (isnan(r10)) r10 = cap;
    q[0] = r10; q[1] = -(r10 + r12); q[2] = r12;
  } else if (r == 2 || r == 3) {
    const float r23 = fmin_nan(P[XB_R23_COEFF] * expf(-f_s * P[XB_DELTA_23] / kt), cap);
    if (r == 2) {
      const float r21 = fmin_nan(expf(logf(r12) - (U_loose - U_t1)), cap);
      q[1] = r21; q[2] = -(r21 + r23); q[3] = r23;
    } else {
      const float r32 = expf(fmin_nan(logf(r23 + 1e-30f) + (U_t2 - U_t1), logf(cap)));
      const float r34 = fmin_nan(P[XB_R34_COEFF] * expf(f_s * P[XB_DELTA_34] / kt), cap);
      q[2] = r32; q[3] = -(r32 + r34); q[4] = r34;
    }
  } else if (r == 4) {
    const float r43 = 0.f, r40 = P[XB_R40];
    q[0] = r40; q[3] = r43; q[4] = -(r43 + r40);
  } else {
    const float k0 = P[XB_SRX_K0], kmax = P[XB_SRX_KMAX], b = P[XB_SRX_B], ca50 = P[XB_SRX_CA50];
    const float cab = powf(ca, b);
    const float r50 = k0 + ((kmax - k0) * cab) / (powf(ca50, b) + cab);
    q[0] = r50; q[5] = -r50;
  }
}

}  // namespace mf
