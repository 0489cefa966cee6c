// Rate matrices and the binned Pade(6,6) matrix exponential.
//
// Restates kernels/transitions.py:99-190 (expm_pade6_batch),
// :434-513 (27 tropomyosin generators), :632-804 (crossbridge generator) with
// the rate laws of kernels/rate_functions.py:165-753.  One thread owns one
// matrix: the tables depend only on (params, pCa, lattice spacing, dt), so
// they are built once per condition whenever those inputs are constant and
// once per step otherwise; the squaring phase optionally runs in float64.
#pragma once
#include "mf_common.cuh"

namespace mf {

__constant__ float kPade6B[7] = {1.0f, 1.0f / 2.0f, 1.0f / 9.0f, 1.0f / 72.0f, 1.0f / 1008.0f,
                                 1.0f / 30240.0f, 1.0f / 1209600.0f};

template <int N>
__device__ __forceinline__ void mm(const float* a, const float* b, float* c) {
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int k = 0; k < N; ++k) {
      float s = a[i * N] * b[k];
#pragma unroll
      for (int j = 1; j < N; ++j) s = fmaf(a[i * N + j], b[j * N + k], s);
      c[i * N + k] = s;
    }
}

template <int N>
__device__ __forceinline__ void mm64(const double* a, const double* b, double* c) {
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int k = 0; k < N; ++k) {
      double s = a[i * N] * b[k];
#pragma unroll
      for (int j = 1; j < N; ++j) s = fma(a[i * N + j], b[j * N + k], s);
      c[i * N + k] = s;
    }
}

// exp(A) in place.  Returns the squaring count s.  sq64_from: squarings run in
// float64 when s >= sq64_from (pass a large value to stay in float32).
template <int N>
__device__ int expm_pade6(float* A, int sq64_from) {
  float nrm = 0.f;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    float r = fabsf(A[i * N]);
#pragma unroll
    for (int j = 1; j < N; ++j) r += fabsf(A[i * N + j]);
    nrm = fmaxf(nrm, r);
  }
  int s = (int)ceilf(log2f(nrm / 0.5f + 1e-10f));
  s = s < 0 ? 0 : s;
  const float inv = 1.0f / exp2f((float)s);  // exact power of two
#pragma unroll
  for (int i = 0; i < N * N; ++i) A[i] = A[i] * inv;
  float A2[N * N], A4[N * N], T[N * N];
  mm<N>(A, A, A2);
  mm<N>(A2, A2, A4);
  // V = b0 I + b2 A2 + b4 A4 + b6 A6 ;  U = A (b1 I + b3 A2 + b5 A4)
  float V[N * N], U[N * N];
  mm<N>(A4, A2, T);  // A6
#pragma unroll
  for (int i = 0; i < N * N; ++i) {
    const bool d = (i / N) == (i % N);
    V[i] = (d ? kPade6B[0] : 0.f) + kPade6B[2] * A2[i] + kPade6B[4] * A4[i] + kPade6B[6] * T[i];
    T[i] = (d ? kPade6B[1] : 0.f) + kPade6B[3] * A2[i] + kPade6B[5] * A4[i];
  }
  mm<N>(A, T, U);
  // Solve (V - U) R = (V + U) by LU with partial pivoting (first maximum).
  // Every index is a compile-time constant -- the row exchange is a select on
  // each candidate row -- so the factors stay in registers.
  float L[N * N], R[N * N];
#pragma unroll
  for (int i = 0; i < N * N; ++i) {
    L[i] = V[i] - U[i];
    R[i] = V[i] + U[i];
  }
#pragma unroll
  for (int k = 0; k < N; ++k) {
    int piv = k;
    float best = fabsf(L[k * N + k]);
#pragma unroll
    for (int i = k + 1; i < N; ++i) {
      const float v = fabsf(L[i * N + k]);
      if (v > best) { best = v; piv = i; }
    }
#pragma unroll
    for (int i = k + 1; i < N; ++i) {
      const bool sw = piv == i;
#pragma unroll
      for (int j = 0; j < N; ++j) {
        const float lk = L[k * N + j], li = L[i * N + j];
        L[k * N + j] = sw ? li : lk;
        L[i * N + j] = sw ? lk : li;
        const float rk = R[k * N + j], ri = R[i * N + j];
        R[k * N + j] = sw ? ri : rk;
        R[i * N + j] = sw ? rk : ri;
      }
    }
    const float dkk = L[k * N + k];
#pragma unroll
    for (int i = k + 1; i < N; ++i) {
      const float l = L[i * N + k] / dkk;
#pragma unroll
      for (int j = k + 1; j < N; ++j) L[i * N + j] = L[i * N + j] - l * L[k * N + j];
#pragma unroll
      for (int j = 0; j < N; ++j) R[i * N + j] = R[i * N + j] - l * R[k * N + j];
    }
  }
#pragma unroll
  for (int i = N - 1; i >= 0; --i)
#pragma unroll
    for (int j = 0; j < N; ++j) {
      float acc = R[i * N + j];
#pragma unroll
      for (int m = i + 1; m < N; ++m) acc = acc - L[i * N + m] * A[m * N + j];
      A[i * N + j] = acc / L[i * N + i];
    }
  // square s times (the reference caps the masked loop at 18 trips)
  const int nsq = s < 18 ? s : 18;
  if (nsq >= sq64_from) {
    // float64 squaring.  The Pade result is first renormalised to unit row
    // sums: rounding that moves a row sum off 1 is what 2^s squarings amplify
    // (a float64 squaring of an unrenormalised float32 result keeps ~5e-3 of
    // relative error at s = 16; renormalised, ~3e-6).
    double D[N * N], E[N * N];
#pragma unroll
    for (int i = 0; i < N; ++i) {
      double rs = 0.0;
#pragma unroll
      for (int j = 0; j < N; ++j) rs += (double)A[i * N + j];
#pragma unroll
      for (int j = 0; j < N; ++j) D[i * N + j] = (double)A[i * N + j] / rs;
    }
    for (int q = 0; q < nsq; ++q) {
      mm64<N>(D, D, E);
#pragma unroll
      for (int i = 0; i < N * N; ++i) D[i] = E[i];
    }
#pragma unroll
    for (int i = 0; i < N; ++i) {
      double rs = 0.0;
#pragma unroll
      for (int j = 0; j < N; ++j) rs += D[i * N + j];
#pragma unroll
      for (int j = 0; j < N; ++j) A[i * N + j] = (float)(D[i * N + j] / rs);
    }
  } else {
    for (int q = 0; q < nsq; ++q) {
      mm<N>(A, A, T);
#pragma unroll
      for (int i = 0; i < N * N; ++i) A[i] = T[i];
    }
#pragma unroll
    for (int i = 0; i < N; ++i) {
      float rs = A[i * N];
#pragma unroll
      for (int j = 1; j < N; ++j) rs += A[i * N + j];
#pragma unroll
      for (int j = 0; j < N; ++j) A[i * N + j] = A[i * N + j] / rs;
    }
  }
#pragma unroll
  for (int i = 0; i < N * N; ++i)
    if (isnan(A[i])) A[i] = 1.0f / (float)N;
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

// Tropomyosin generator of configuration cfg = 9*n2 + 3*n3 + n_closed.
static __device__ void tm_generator(const float* P, float pCa, int cfg, float* Q) {
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
#pragma unroll
  for (int i = 0; i < 16; ++i) Q[i] = 0.f;
  Q[0] = -k01; Q[1] = k01;
  Q[4] = k10; Q[5] = -(k10 + k12); Q[6] = k12;
  Q[9] = k21; Q[10] = -(k21 + k23); Q[11] = k23;
  Q[12] = k30; Q[14] = k32; Q[15] = -(k30 + k32);
}

// Crossbridge generator at axial offset x, spacing d, permissiveness perm.
static __device__ void xb_generator(const float* P, float pCa, float x, float d, float perm, float* Q) {
  const float ca = powf(10.0f, -pCa);
  const float r = sqrtf(x * x + d * d);
  const float th = atan2f(d, x);
  const float kt = 1.3810e-23f * (P[TEMP_CELSIUS] + 273.15f) * 1e21f;
  const float gw = r - P[XB_G_REST_WEAK], cw = th - P[XB_C_REST_WEAK];
  const float gs = r - P[XB_G_REST_STRONG], cs = th - P[XB_C_REST_STRONG];
  const float Ew = (0.5f * P[XB_G_K_WEAK] * (gw * gw) + 0.5f * P[XB_C_K_WEAK] * (cw * cw)) / kt;
  const float Es = (0.5f * P[XB_G_K_STRONG] * (gs * gs) + 0.5f * P[XB_C_K_STRONG] * (cs * cs)) / kt;
  const float Ediff = Ew - Es;
  const float U_drx = P[XB_U_DRX];
  const float U_loose = P[XB_U_LOOSE] + Ew;
  const float U_t1 = P[XB_U_TIGHT_1] + Es;
  const float U_t2 = P[XB_U_TIGHT_2] + Es;
  const float f_s = P[XB_G_K_STRONG] * gs + (1.0f / r) * P[XB_C_K_STRONG] * cs;
  const float cap = 10000.0f;
  float r01 = perm * P[XB_R01_COEFF] * expf(-Ew);
  if (isnan(r01)) r01 = 0.f;
  float r10 = fmin_nan(expf(logf(r01 + 0.005f) - (U_drx - U_loose)), cap);
  if (isnan(r10)) r10 = cap;
  float r12 = P[XB_R12_COEFF] * expf(fmin_nan(Ediff, 30.0f) / 2.0f);
  if (isnan(r12)) r12 = 0.f;
  const float r21 = fmin_nan(expf(logf(r12) - (U_loose - U_t1)), cap);
  const float r23 = fmin_nan(P[XB_R23_COEFF] * expf(-f_s * P[XB_DELTA_23] / kt), cap);
  const float r32 = expf(fmin_nan(logf(r23 + 1e-30f) + (U_t2 - U_t1), logf(cap)));
  const float r34 = fmin_nan(P[XB_R34_COEFF] * expf(f_s * P[XB_DELTA_34] / kt), cap);
  const float r43 = 0.f;
  const float r40 = P[XB_R40], r04 = P[XB_R04], r05 = P[XB_R05];
  const float k0 = P[XB_SRX_K0], kmax = P[XB_SRX_KMAX], b = P[XB_SRX_B], ca50 = P[XB_SRX_CA50];
  const float cab = powf(ca, b);
  const float r50 = k0 + ((kmax - k0) * cab) / (powf(ca50, b) + cab);
#pragma unroll
  for (int i = 0; i < 36; ++i) Q[i] = 0.f;
  Q[0] = -(r01 + r04 + r05); Q[1] = r01; Q[4] = r04; Q[5] = r05;
  Q[6] = r10; Q[7] = -(r10 + r12); Q[8] = r12;
  Q[13] = r21; Q[14] = -(r21 + r23); Q[15] = r23;
  Q[20] = r32; Q[21] = -(r32 + r34); Q[22] = r34;
  Q[24] = r40; Q[27] = r43; Q[28] = -(r43 + r40);
  Q[30] = r50; Q[35] = -r50;
}

}  // namespace mf
