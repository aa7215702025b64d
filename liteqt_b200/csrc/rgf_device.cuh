// rgf_device.cuh -- block-level building blocks of the FP64 RGF kernels.
//
// Every routine here is executed cooperatively by all kThreads threads of one
// CTA on nb x nb complex blocks stored column-major with leading dimension nb
// (element (i,j) at i + j*nb, interleaved re/im as double2 -- the complex(8)
// layout of the Fortran caller).  Pointers are generic: a block may live in
// shared memory or in global memory (L1/L2 cached).
//
// The dense products run on the FP64 tensor pipe: mma.sync m8n8k4 f64
// (DMMA), four real products per complex product.  On B200 the DMMA and DFMA
// peaks are equal (about 37 TFLOP/s), but DMMA issues 256 FMAs per
// instruction, which leaves the issue slots to the operand loads.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "rgf_internal.h"

namespace rgf {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

// ---------------------------------------------------------------- complex
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__device__ __forceinline__ double2 czero() { return make_double2(0.0, 0.0); }
// 1/(a+ib) = (a-ib) / (a^2+b^2).  a and b are first scaled by the power of
// two 2^-e (exact) that brings max(|a|, |b|) into [1/2, 1), so the squares
// neither overflow nor underflow, and one division forms 1/(a^2+b^2).  Zero,
// subnormal, infinite and NaN arguments and exponents near the ends of the
// range take the quotient form with two divisions.
__device__ __forceinline__ double2 crecip(double2 a) {
  const double s = fmax(fabs(a.x), fabs(a.y));
  const int e = (int)((__double_as_longlong(s) >> 52) & 0x7ff) - 1022;  // s in [2^(e-1), 2^e)
  if (e < -1020 || e > 1020) {
    const double ar = a.x / s, ai = a.y / s;
    const double d = ar * ar + ai * ai;
    return make_double2(ar / (d * s), -ai / (d * s));
  }
  const double sc = __longlong_as_double((long long)(1023 - e) << 52);  // 2^-e
  const double ar = a.x * sc, ai = a.y * sc;
  const double r = 1.0 / (ar * ar + ai * ai);
  return make_double2(ar * r * sc, -ai * r * sc);
}
// |re| + |im|: the pivot measure of LAPACK's izamax (dcabs1), used by zgetrf.
__device__ __forceinline__ double cabs1(double2 a) { return fabs(a.x) + fabs(a.y); }

__device__ __forceinline__ double fermi(double a) { return 1.0 / (1.0 + exp(a)); }

// ---------------------------------------------------------------- DMMA
// D(8x8) += A(8x4, row) * B(4x8, col); lane (g = lane/4, t = lane%4) holds
// a = A[g][t], b = B[t][g], d = D[g][2t], D[g][2t+1].
__device__ __forceinline__ void dmma884(double& d0, double& d1, double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
      : "+d"(d0), "+d"(d1)
      : "d"(a), "d"(b));
}

// D(16x8) += A(16x4, row) * B(4x8, col); lane (g, t) holds a0 = A[g][t],
// a1 = A[g+8][t], b = B[t][g], d0, d1 = D[g][2t, 2t+1], d2, d3 = D[g+8][2t,
// 2t+1]: two m8n8k4 products sharing B in one instruction.
__device__ __forceinline__ void dmma1684(double& d0, double& d1, double& d2, double& d3, double a0,
                                         double a1, double b) {
  asm("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};"
      : "+d"(d0), "+d"(d1), "+d"(d2), "+d"(d3)
      : "d"(a0), "d"(a1), "d"(b));
}

// ---------------------------------------------------------------- reductions
struct SmemRed {
  double v[2 * kWarps];
};

// Sum over the CTA; every thread gets the same value (fixed order).
__device__ __forceinline__ double2 block_sum2(double2 v, SmemRed& r) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
  }
  if (lane == 0) { r.v[2 * warp] = v.x; r.v[2 * warp + 1] = v.y; }
  __syncthreads();
  double2 s = czero();
#pragma unroll
  for (int w = 0; w < kWarps; w++) { s.x += r.v[2 * w]; s.y += r.v[2 * w + 1]; }
  __syncthreads();
  return s;
}

// ---------------------------------------------------------------- elementwise
// body(i, j, idx) over every element of an n x n block.
template <class F>
__device__ __forceinline__ void for_each_elem(int n, F&& body) {
  const int n2 = n * n;
  for (int idx = threadIdx.x; idx < n2; idx += kThreads) {
    const int j = idx / n, i = idx - j * n;
    body(i, j, idx);
  }
}

// One complex 8x8x4 step on TM x TN subtiles: Cr += Ar Br - Ai Bi,
// Ci += Ar Bi + Ai Br as four rounds of real DMMAs, each round over all
// subtiles, so that consecutive MMAs on one accumulator are TM*TN apart.
template <int TM, int TN>
__device__ __forceinline__ void cmma_step(double (&cr)[TM][TN][2], double (&ci)[TM][TN][2],
                                          const double2 (&av)[TM], const double2 (&bv)[TN],
                                          double a_sg, double b_sg) {
  if constexpr (TM % 2 == 0) {
    // row subtiles (2p, 2p+1) are rows g and g+8 of one 16-row tile
#pragma unroll
    for (int p = 0; p < TM / 2; p++)
#pragma unroll
      for (int b = 0; b < TN; b++)
        dmma1684(cr[2 * p][b][0], cr[2 * p][b][1], cr[2 * p + 1][b][0], cr[2 * p + 1][b][1],
                 av[2 * p].x, av[2 * p + 1].x, bv[b].x);
#pragma unroll
    for (int p = 0; p < TM / 2; p++)
#pragma unroll
      for (int b = 0; b < TN; b++)
        dmma1684(ci[2 * p][b][0], ci[2 * p][b][1], ci[2 * p + 1][b][0], ci[2 * p + 1][b][1],
                 av[2 * p].x, av[2 * p + 1].x, bv[b].y * b_sg);
#pragma unroll
    for (int p = 0; p < TM / 2; p++)
#pragma unroll
      for (int b = 0; b < TN; b++)
        dmma1684(cr[2 * p][b][0], cr[2 * p][b][1], cr[2 * p + 1][b][0], cr[2 * p + 1][b][1],
                 -av[2 * p].y * a_sg, -av[2 * p + 1].y * a_sg, bv[b].y * b_sg);
#pragma unroll
    for (int p = 0; p < TM / 2; p++)
#pragma unroll
      for (int b = 0; b < TN; b++)
        dmma1684(ci[2 * p][b][0], ci[2 * p][b][1], ci[2 * p + 1][b][0], ci[2 * p + 1][b][1],
                 av[2 * p].y * a_sg, av[2 * p + 1].y * a_sg, bv[b].x);
  } else {
#pragma unroll
    for (int a = 0; a < TM; a++)
#pragma unroll
      for (int b = 0; b < TN; b++) dmma884(cr[a][b][0], cr[a][b][1], av[a].x, bv[b].x);
#pragma unroll
    for (int a = 0; a < TM; a++)
#pragma unroll
      for (int b = 0; b < TN; b++) dmma884(ci[a][b][0], ci[a][b][1], av[a].x, bv[b].y * b_sg);
#pragma unroll
    for (int a = 0; a < TM; a++)
#pragma unroll
      for (int b = 0; b < TN; b++) dmma884(cr[a][b][0], cr[a][b][1], -av[a].y * a_sg, bv[b].y * b_sg);
#pragma unroll
    for (int a = 0; a < TM; a++)
#pragma unroll
      for (int b = 0; b < TN; b++) dmma884(ci[a][b][0], ci[a][b][1], av[a].y * a_sg, bv[b].x);
  }
}

// ---------------------------------------------------------------- GEMM
// C = op(A) * op(B) for n x n complex blocks, op = identity or conjugate
// transpose (cA / cB).  The result is not stored: epi(i, j, value) is called
// exactly once per output element, by the thread that owns it, so an epilogue
// may read-modify-write C[i + j*n] (accumulation) or write several outputs.
// n must be a multiple of 8*TM and 8*TN.  The caller synchronises.
template <int TM, int TN, class Epi>
__device__ __forceinline__ void cgemm(int n, const double2* A, bool cA, const double2* B, bool cB,
                                      Epi&& epi) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int gm = n / (8 * TM), gn = n / (8 * TN);
  // strides of op(A)[i][k] and op(B)[k][j] in memory
  const int a_si = cA ? n : 1, a_sk = cA ? 1 : n;
  const int b_sk = cB ? n : 1, b_sj = cB ? 1 : n;
  const double a_sg = cA ? -1.0 : 1.0, b_sg = cB ? -1.0 : 1.0;
  for (int grp = warp; grp < gm * gn; grp += kWarps) {
    const int m0 = (grp % gm) * (8 * TM), n0 = (grp / gm) * (8 * TN);
    double cr[TM][TN][2], ci[TM][TN][2];
#pragma unroll
    for (int a = 0; a < TM; a++)
#pragma unroll
      for (int b = 0; b < TN; b++) { cr[a][b][0] = cr[a][b][1] = ci[a][b][0] = ci[a][b][1] = 0.0; }
    const double2* Ap[TM];
    const double2* Bp[TN];
#pragma unroll
    for (int a = 0; a < TM; a++) Ap[a] = A + (m0 + 8 * a + g) * a_si + t * a_sk;
#pragma unroll
    for (int b = 0; b < TN; b++) Bp[b] = B + t * b_sk + (n0 + 8 * b + g) * b_sj;
#pragma unroll 4
    for (int k0 = 0; k0 < n; k0 += 4) {
      double2 av[TM], bv[TN];
#pragma unroll
      for (int a = 0; a < TM; a++) av[a] = Ap[a][k0 * a_sk];
#pragma unroll
      for (int b = 0; b < TN; b++) bv[b] = Bp[b][k0 * b_sk];
      cmma_step<TM, TN>(cr, ci, av, bv, a_sg, b_sg);
    }
#pragma unroll
    for (int a = 0; a < TM; a++)
#pragma unroll
      for (int b = 0; b < TN; b++)
#pragma unroll
        for (int c = 0; c < 2; c++)
          epi(m0 + 8 * a + g, n0 + 8 * b + 2 * t + c, make_double2(cr[a][b][c], ci[a][b][c]));
  }
}

// ---------------------------------------------------------------- inverse
// Pivot bookkeeping of the inverse (the row / column vectors of the current
// elimination step live in dynamic shared memory, see gj_invert).
struct SmemInv {
  int16_t perm[kMaxNb];
  int16_t colsrc[kMaxNb];
  int16_t coldst[kMaxNb];  // inverse of colsrc (blocked inverse)
  int16_t rmap[kMaxNb];  // row map of the current panel (outside the GEMM staging area)
  double2 pivval;
  double2 akc;  // the pivot column's entry in row k before the interchange
  int piv;
  int singular;
};

// In-place Gauss-Jordan inversion with partial (row) pivoting of the n x n
// block X, then dst[:, j] = X[:, colsrc[j]] to undo the row interchanges
// (and the same into dst2 if non-null).  Pivot: largest |re|+|im| in the
// column, first index on ties, as LAPACK zgetrf.  A zero pivot makes the
// result the zero block (the reference's `invert` fallback,
// green_rgf.f90:4429-4437) and the return value 1.
// Preconditions: X holds the matrix and is visible to all threads.
// rowk, fcol: shared scratch of n complex values each.
__device__ __noinline__ static int gj_invert(int n, double2* X, double2* dst, double2* dst2, SmemInv& s,
                                             double2* rowk, double2* fcol) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) s.singular = 0;
  for (int k = 0; k < n; k++) {
    if (warp == 0) {
      double best = -1.0;
      int bi = k;
      for (int i = k + lane; i < n; i += 32) {
        const double v = cabs1(X[i + k * n]);
        if (v > best) { best = v; bi = i; }
      }
#pragma unroll
      for (int o = 16; o; o >>= 1) {
        const double ob = __shfl_xor_sync(0xffffffffu, best, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
      }
      if (lane == 0) {
        s.piv = bi;
        s.pivval = X[bi + k * n];
        s.perm[k] = (int16_t)bi;
        if (best == 0.0) s.singular = 1;
      }
    }
    __syncthreads();
    if (s.singular) break;  // uniform
    const int p = s.piv;
    const double2 pinv = crecip(s.pivval);
    // swap rows k and p, scale the new row k; X[k][k] becomes 1/pivot
    for (int j = tid; j < n; j += kThreads) {
      const double2 a = X[k + j * n];
      const double2 b = X[p + j * n];
      if (p != k) X[p + j * n] = a;
      const double2 r = (j == k) ? pinv : cmul(b, pinv);
      X[k + j * n] = r;
      rowk[j] = r;
    }
    __syncthreads();
    for (int i = tid; i < n; i += kThreads) fcol[i] = (i == k) ? czero() : X[i + k * n];
    __syncthreads();
    // X[i][j] -= f_i * rowk[j] for i != k, with X[i][k] treated as 0
    for_each_elem(n, [&](int i, int j, int idx) {
      if (i == k) return;
      const double2 f = fcol[i];
      const double2 x = (j == k) ? czero() : X[idx];
      const double2 r = rowk[j];
      X[idx] = make_double2(x.x - (f.x * r.x - f.y * r.y), x.y - (f.x * r.y + f.y * r.x));
    });
    __syncthreads();
  }
  const int sing = s.singular;
  if (sing) {
    for_each_elem(n, [&](int, int, int idx) {
      dst[idx] = czero();
      if (dst2) dst2[idx] = czero();
    });
    __syncthreads();
    return 1;
  }
  if (tid == 0) {
    for (int j = 0; j < n; j++) s.colsrc[j] = (int16_t)j;
    for (int k = n - 1; k >= 0; k--) {
      const int q = s.perm[k];
      if (q != k) { const int16_t tmp = s.colsrc[k]; s.colsrc[k] = s.colsrc[q]; s.colsrc[q] = tmp; }
    }
  }
  __syncthreads();
  for_each_elem(n, [&](int i, int j, int idx) {
    const double2 v = X[i + s.colsrc[j] * n];
    dst[idx] = v;
    if (dst2) dst2[idx] = v;
  });
  __syncthreads();
  return 0;
}

// Re/Im of Tr[A * B] = sum_{i,k} A[i][k] B[k][i] (only the diagonal of the
// product is formed).  opB_plus: B = B1 + (B2 - B2^H) when B2 is non-null.
__device__ __forceinline__ double2 trace_prod(int n, const double2* A, const double2* B, SmemRed& r) {
  double2 acc = czero();
  for_each_elem(n, [&](int i, int k, int idx) { acc = cadd(acc, cmul(A[idx], B[k + i * n])); });
  return block_sum2(acc, r);
}

}  // namespace rgf
