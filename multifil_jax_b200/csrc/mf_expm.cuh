// Rate matrices and the binned Pade(6,6) matrix exponential.
//
// Restates kernels/transitions.py:99-190 (expm_pade6_batch),
// :434-513 (27 tropomyosin generators), :632-804 (crossbridge generator) with
// the rate laws of kernels/rate_functions.py:165-753.  The tables depend only
// on (params, pCa, lattice spacing, dt), so they are built once per condition
// whenever those inputs are constant and once per step otherwise.
//
// One matrix is owned by a pair of consecutive lanes: lane h of the pair
// holds rows h*N/2 .. h*N/2 + N/2 - 1.  Products, the pivot search, the row
// exchanges and the back substitution move rows between the two lanes with
// width-2 shuffles, so a lane holds half a matrix of registers (a whole 6x6
// float64 product in one thread does not fit the register budget and
// spills), and sixteen matrices of a warp advance together.  The squaring
// phase optionally runs in float64.
#pragma once
#include "mf_common.cuh"

namespace mf {

__constant__ float kPade6B[7] = {1.0f, 1.0f / 2.0f, 1.0f / 9.0f, 1.0f / 72.0f, 1.0f / 1008.0f,
                                 1.0f / 30240.0f, 1.0f / 1209600.0f};

constexpr int kPair = 2;  // lanes per matrix

// This lane's rows of C = A B, from its rows of A (a) and the rows of B held
// by the pair (b): C[i][k] = A[i][0] B[0][k] + ... in increasing j, one fused
// multiply-add per further term.  A lane already holds its own rows of B;
// the partner's rows are swapped in once with an xor shuffle (R N values per
// product, half of what a broadcast of every row moves: the shuffle unit
// issues one warp instruction per clock per SM and bounds this code).  Done
// in blocks of R columns so that only R x R swapped values are live.
template <int N, class F>
__device__ __forceinline__ void mm_pair(unsigned pmask, int h, const F (&a)[N / 2][N], const F (&b)[N / 2][N],
                                        F (&c)[N / 2][N]) {
  constexpr int R = N / 2;
#pragma unroll
  for (int k0 = 0; k0 < N; k0 += R) {
    F o[R][R];  // the partner's rows of B, columns k0 .. k0 + R - 1
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int kk = 0; kk < R; ++kk) o[r][kk] = __shfl_xor_sync(pmask, b[r][k0 + kk], 1, kPair);
#pragma unroll
    for (int j = 0; j < N; ++j) {
      const bool own = j / R == h;
#pragma unroll
      for (int kk = 0; kk < R; ++kk) {
        const F bj = own ? b[j % R][k0 + kk] : o[j % R][kk];
#pragma unroll
        for (int i = 0; i < R; ++i)
          c[i][k0 + kk] = j == 0 ? a[i][0] * bj : fma(a[i][j], bj, c[i][k0 + kk]);
      }
    }
  }
}

// Row `row` of a pair's matrix (runtime row index), fetched by both lanes.
template <int N, class F>
__device__ __forceinline__ void fetch_row(unsigned pmask, const F (&m)[N / 2][N], int row, F (&out)[N]) {
  constexpr int R = N / 2;
  const int li = row % R;
#pragma unroll
  for (int k = 0; k < N; ++k) {
    F v = m[0][k];
#pragma unroll
    for (int i = 1; i < R; ++i) v = li == i ? m[i][k] : v;
    out[k] = __shfl_sync(pmask, v, row / R, kPair);
  }
}

// exp(A) of the pair's matrix, this lane's rows in a[][] (in place).
// Returns the squaring count s (2^s >= ||A||_inf / 0.5).  sq64_from: the
// squarings run in float64 when s >= sq64_from (a large value keeps them in
// float32).  Both lanes of the pair take part (pmask names the pair).
template <int N>
__device__ int expm_pair(unsigned pmask, int h, float (&a)[N / 2][N], int sq64_from) {
  constexpr int R = N / 2;
  // infinity norm: the largest absolute row sum (NaN-propagating, as jnp.max)
  float nrm = 0.f;
#pragma unroll
  for (int i = 0; i < R; ++i) {
    float rs = fabsf(a[i][0]);
#pragma unroll
    for (int j = 1; j < N; ++j) rs += fabsf(a[i][j]);
    nrm = fmax_nan(nrm, rs);
  }
  nrm = fmax_nan(nrm, __shfl_xor_sync(pmask, nrm, 1, kPair));
  int s = (int)ceilf(log2f(nrm / 0.5f + 1e-10f));
  s = s < 0 ? 0 : s;
  const float inv = 1.0f / exp2f((float)s);  // exact power of two
#pragma unroll
  for (int i = 0; i < R; ++i)
#pragma unroll
    for (int j = 0; j < N; ++j) a[i][j] = a[i][j] * inv;
  // V = b0 I + b2 A2 + b4 A4 + b6 A6 ;  U = A (b1 I + b3 A2 + b5 A4), in an
  // order that keeps at most four half-matrices live
  float a2[R][N], a4[R][N], t[R][N], u[R][N];
  mm_pair<N>(pmask, h, a, a, a2);
  mm_pair<N>(pmask, h, a2, a2, a4);
#pragma unroll
  for (int i = 0; i < R; ++i)
#pragma unroll
    for (int j = 0; j < N; ++j)
      t[i][j] = (j == h * R + i ? kPade6B[1] : 0.f) + kPade6B[3] * a2[i][j] + kPade6B[5] * a4[i][j];
  mm_pair<N>(pmask, h, a, t, u);
  mm_pair<N>(pmask, h, a4, a2, t);  // A6
  // Solve (V - U) X = (V + U) by LU with partial pivoting (the first row of
  // largest magnitude in the column is the pivot).  L reuses a2, R reuses a4.
#pragma unroll
  for (int i = 0; i < R; ++i)
#pragma unroll
    for (int j = 0; j < N; ++j) {
      const float v = (j == h * R + i ? kPade6B[0] : 0.f) + kPade6B[2] * a2[i][j] + kPade6B[4] * a4[i][j] +
                      kPade6B[6] * t[i][j];
      a2[i][j] = v - u[i][j];
      a4[i][j] = v + u[i][j];
    }
  float (&L)[R][N] = a2;
  float (&Rm)[R][N] = a4;
  // Rows k .. N-1 of the last R columns are lane 1's alone, so those steps
  // (and the first R steps of the back substitution, lane 0's alone) need no
  // shuffles; a pivot that stays on the diagonal (the usual case: the scaled
  // V - U is close to I) needs one broadcast of the pivot row and no exchange.
#pragma unroll
  for (int k = 0; k < N; ++k) {
    // pivot: largest |L[i][k]| over rows i >= k, lowest index on ties
    float best = -2.f;
    int piv = N;
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const int gi = h * R + i;
      float v = fabsf(L[i][k]);
      if (v != v) v = -1.f;
      if (gi >= k && v > best) { best = v; piv = gi; }
    }
    if (k < R) {  // candidates in both lanes
      const float ob = __shfl_xor_sync(pmask, best, 1, kPair);
      const int op = __shfl_xor_sync(pmask, piv, 1, kPair);
      if (ob > best || (ob == best && op < piv)) { best = ob; piv = op; }
    }
    if (piv >= N) piv = k;
    // exchange rows k and piv; Lp, Rp: the pivot row
    float Lp[N], Rp[N];
    if (k >= R) {  // both rows are lane 1's (lane 0 has no row >= k and changes nothing)
      const int li = piv % R;
#pragma unroll
      for (int j = 0; j < N; ++j) {
        float vl = L[0][j], vr = Rm[0][j];
#pragma unroll
        for (int i = 1; i < R; ++i) {
          vl = li == i ? L[i][j] : vl;
          vr = li == i ? Rm[i][j] : vr;
        }
        Lp[j] = vl;
        Rp[j] = vr;
      }
      if (h == k / R && piv != k) {
#pragma unroll
        for (int i = 0; i < R; ++i) {
          if (h * R + i == piv) {
#pragma unroll
            for (int j = 0; j < N; ++j) { L[i][j] = L[k % R][j]; Rm[i][j] = Rm[k % R][j]; }
          }
        }
#pragma unroll
        for (int j = 0; j < N; ++j) { L[k % R][j] = Lp[j]; Rm[k % R][j] = Rp[j]; }
      }
    } else if (piv == k) {  // pair-uniform: row k stays, lane 0 broadcasts it
#pragma unroll
      for (int j = 0; j < N; ++j) {
        Lp[j] = __shfl_sync(pmask, L[k % R][j], k / R, kPair);
        Rp[j] = __shfl_sync(pmask, Rm[k % R][j], k / R, kPair);
      }
    } else {
      float Lk[N], Rk[N];
      fetch_row<N>(pmask, L, piv, Lp);
      fetch_row<N>(pmask, Rm, piv, Rp);
#pragma unroll
      for (int j = 0; j < N; ++j) {
        Lk[j] = __shfl_sync(pmask, L[k % R][j], k / R, kPair);
        Rk[j] = __shfl_sync(pmask, Rm[k % R][j], k / R, kPair);
      }
#pragma unroll
      for (int i = 0; i < R; ++i) {
        if (h * R + i == piv) {
#pragma unroll
          for (int j = 0; j < N; ++j) { L[i][j] = Lk[j]; Rm[i][j] = Rk[j]; }
        }
      }
      if (h == k / R) {
#pragma unroll
        for (int j = 0; j < N; ++j) { L[k % R][j] = Lp[j]; Rm[k % R][j] = Rp[j]; }
      }
    }
    // eliminate below the pivot with the pivot row (now Lp, Rp)
#pragma unroll
    for (int i = 0; i < R; ++i) {
      if (h * R + i > k) {
        const float l = L[i][k] / Lp[k];
#pragma unroll
        for (int j = k + 1; j < N; ++j) L[i][j] = L[i][j] - l * Lp[j];
#pragma unroll
        for (int j = 0; j < N; ++j) Rm[i][j] = Rm[i][j] - l * Rp[j];
      }
    }
  }
  // back substitution, last row first: X[i] = (R[i] - sum_{m>i} L[i][m] X[m]) / L[i][i]
#pragma unroll
  for (int g = N - 1; g >= 0; --g) {
    if (h == g / R) {
#pragma unroll
      for (int j = 0; j < N; ++j) a[g % R][j] = Rm[g % R][j] / L[g % R][g];
    }
    float xg[N];
    if (g >= R) {  // lane 0's rows (all < g) need lane 1's row g
#pragma unroll
      for (int j = 0; j < N; ++j) xg[j] = __shfl_sync(pmask, a[g % R][j], g / R, kPair);
    } else {       // rows < g are lane 0's, which holds row g
#pragma unroll
      for (int j = 0; j < N; ++j) xg[j] = a[g % R][j];
    }
#pragma unroll
    for (int i = 0; i < R; ++i) {
      if (h * R + i < g) {
#pragma unroll
        for (int j = 0; j < N; ++j) Rm[i][j] = Rm[i][j] - L[i][g] * xg[j];
      }
    }
  }
  // square s times (the reference caps the masked loop at 18 trips)
  const int nsq = s < 18 ? s : 18;
  if (nsq >= sq64_from) {
    // float64 squaring.  The Pade rows are first renormalised to unit sums:
    // rounding that moves a row sum off 1 is what 2^s squarings amplify (a
    // float64 squaring of an unrenormalised float32 result keeps ~5e-3 of
    // relative error at s = 16; renormalised, ~3e-6).
    double D[R][N], E[R][N];
#pragma unroll
    for (int i = 0; i < R; ++i) {
      double sum = 0.0;
#pragma unroll
      for (int j = 0; j < N; ++j) sum += (double)a[i][j];
#pragma unroll
      for (int j = 0; j < N; ++j) D[i][j] = (double)a[i][j] / sum;
    }
    for (int q = 0; q < nsq; ++q) {
      mm_pair<N>(pmask, h, D, D, E);
#pragma unroll
      for (int i = 0; i < R; ++i)
#pragma unroll
        for (int j = 0; j < N; ++j) D[i][j] = E[i][j];
    }
#pragma unroll
    for (int i = 0; i < R; ++i) {
      double sum = 0.0;
#pragma unroll
      for (int j = 0; j < N; ++j) sum += D[i][j];
#pragma unroll
      for (int j = 0; j < N; ++j) a[i][j] = (float)(D[i][j] / sum);
    }
  } else {
    float c[R][N];
    for (int q = 0; q < nsq; ++q) {
      mm_pair<N>(pmask, h, a, a, c);
#pragma unroll
      for (int i = 0; i < R; ++i)
#pragma unroll
        for (int j = 0; j < N; ++j) a[i][j] = c[i][j];
    }
#pragma unroll
    for (int i = 0; i < R; ++i) {
      float sum = a[i][0];
#pragma unroll
      for (int j = 1; j < N; ++j) sum += a[i][j];
#pragma unroll
      for (int j = 0; j < N; ++j) a[i][j] = a[i][j] / sum;
    }
  }
#pragma unroll
  for (int i = 0; i < R; ++i)
#pragma unroll
    for (int j = 0; j < N; ++j)
      if (isnan(a[i][j])) a[i][j] = 1.0f / (float)N;
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

// Rows 2h, 2h+1 of the tropomyosin generator of configuration
// cfg = 9*n2 + 3*n3 + n_closed (Ising coupling h; forward rates x e^{h/2},
// backward x e^{-h/2}).
static __device__ void tm_generator_rows(const float* P, float pCa, int cfg, int h, float (&q)[2][4]) {
  const float ca = powf(10.0f, -pCa);
  const float n2 = (float)(cfg / 9), n3 = (float)((cfg / 3) % 3), nc = (float)(cfg % 3);
  const float JC = P[TM_J_C], JM = P[TM_J_M];
  const float hh = JC * n2 + JM * n3 - 0.5f * (JC + JM) * nc;
  const float fwd = expf(0.5f * hh), bwd = expf(-0.5f * hh);
  const float k01 = P[TM_K_01] * ca * fwd;
  const float k12 = P[TM_K_12] * fwd;
  const float k23 = P[TM_K_23] * fwd;
  const float k30 = P[TM_K_30];
  const float k10 = (P[TM_K_01] / P[TM_KEQ_01]) * bwd;
  const float k21 = (P[TM_K_12] / P[TM_KEQ_12]) * bwd;
  const float k32 = (P[TM_K_23] / P[TM_KEQ_23]) * bwd;
  if (h == 0) {
    q[0][0] = -k01; q[0][1] = k01; q[0][2] = 0.f; q[0][3] = 0.f;
    q[1][0] = k10; q[1][1] = -(k10 + k12); q[1][2] = k12; q[1][3] = 0.f;
  } else {
    q[0][0] = 0.f; q[0][1] = k21; q[0][2] = -(k21 + k23); q[0][3] = k23;
    q[1][0] = k30; q[1][1] = 0.f; q[1][2] = k32; q[1][3] = -(k30 + k32);
  }
}

// Rows 3h .. 3h+2 of the crossbridge generator at axial offset x, spacing
// d, permissiveness perm.
static __device__ void xb_generator_rows(const float* P, float pCa, float x, float d, float perm, int h,
                                         float (&q)[3][6]) {
  const float ca = powf(10.0f, -pCa);
  const float rr = sqrtf(x * x + d * d);
  const float th = atan2f(d, x);
  const float kt = 1.3810e-23f * (P[TEMP_CELSIUS] + 273.15f) * 1e21f;
  const float gw = rr - P[XB_G_REST_WEAK], cw = th - P[XB_C_REST_WEAK];
  const float gs = rr - P[XB_G_REST_STRONG], cs = th - P[XB_C_REST_STRONG];
  const float Ew = (0.5f * P[XB_G_K_WEAK] * (gw * gw) + 0.5f * P[XB_C_K_WEAK] * (cw * cw)) / kt;
  const float Es = (0.5f * P[XB_G_K_STRONG] * (gs * gs) + 0.5f * P[XB_C_K_STRONG] * (cs * cs)) / kt;
  const float U_loose = P[XB_U_LOOSE] + Ew;
  const float U_t1 = P[XB_U_TIGHT_1] + Es;
  const float f_s = P[XB_G_K_STRONG] * gs + (1.0f / rr) * P[XB_C_K_STRONG] * cs;
  const float cap = 10000.0f;
  const float r23 = fmin_nan(P[XB_R23_COEFF] * expf(-f_s * P[XB_DELTA_23] / kt), cap);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 6; ++j) q[i][j] = 0.f;
  if (h == 0) {
    const float Ediff = Ew - Es;
    const float U_drx = P[XB_U_DRX];
    float r01 = perm * P[XB_R01_COEFF] * expf(-Ew);
    if (isnan(r01)) r01 = 0.f;
    float r10 = fmin_nan(expf(logf(r01 + 0.005f) - (U_drx - U_loose)), cap);
    if (isnan(r10)) r10 = cap;
    float r12 = P[XB_R12_COEFF] * expf(fmin_nan(Ediff, 30.0f) / 2.0f);
    if (isnan(r12)) r12 = 0.f;
    const float r21 = fmin_nan(expf(logf(r12) - (U_loose - U_t1)), cap);
    const float r04 = P[XB_R04], r05 = P[XB_R05];
    q[0][0] = -(r01 + r04 + r05); q[0][1] = r01; q[0][4] = r04; q[0][5] = r05;
    q[1][0] = r10; q[1][1] = -(r10 + r12); q[1][2] = r12;
    q[2][1] = r21; q[2][2] = -(r21 + r23); q[2][3] = r23;
  } else {
    const float U_t2 = P[XB_U_TIGHT_2] + Es;
    const float r32 = expf(fmin_nan(logf(r23 + 1e-30f) + (U_t2 - U_t1), logf(cap)));
    const float r34 = fmin_nan(P[XB_R34_COEFF] * expf(f_s * P[XB_DELTA_34] / kt), cap);
    const float r43 = 0.f, r40 = P[XB_R40];
    const float k0 = P[XB_SRX_K0], kmax = P[XB_SRX_KMAX], b = P[XB_SRX_B], ca50 = P[XB_SRX_CA50];
    const float cab = powf(ca, b);
    const float r50 = k0 + ((kmax - k0) * cab) / (powf(ca50, b) + cab);
    q[0][2] = r32; q[0][3] = -(r32 + r34); q[0][4] = r34;
    q[1][0] = r40; q[1][3] = r43; q[1][4] = -(r43 + r40);
    q[2][0] = r50; q[2][5] = -r50;
  }
}

}  // namespace mf
