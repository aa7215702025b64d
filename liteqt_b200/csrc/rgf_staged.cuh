// rgf_staged.cuh -- shared-memory-staged complex DMMA GEMM and blocked
// Gauss-Jordan inverse for the block sizes the benchmarks use
// (nb = 32, 64, 128, 256).
//
// GEMM: C(M x N) = op(A)(M x K) * op(B)(K x N), complex FP64, operands in
// global memory (column-major with leading dimensions lda / ldb), op = N or
// C (conjugate transpose).  The CTA walks output tiles of PM x PN; for each
// it streams K in chunks of KC through two shared-memory stages filled with
// cp.async (16-byte copies, one complex value each), while the 8 warps run
// mma.sync.m8n8k4.f64 on the other stage.  Shared tiles are k-major with a
// row pitch of PM + 2 complex values, which makes the fragment reads of a
// quarter warp (rows g = 0,1 x k = 0..3) hit 8 distinct 16-byte bank groups.
//
// Inverse (nb >= 128): Gauss-Jordan with partial row pivoting, blocked by
// panels of PW columns.  Each panel is eliminated unblocked in shared memory
// (pivot rule: largest |re|+|im|, first index on ties, as zgetrf), its row
// interchanges are applied to the other columns, and the other columns get
// the panel's transformation as one rank-PW GEMM update:
//     rows of the panel:  X[P, j] = U[P, :] R[:, j]
//     other rows:         X[i, j] = X[i, j] + U[i, :] R[:, j]
// with U the eliminated panel and R = X[P, :] before the update.  The pivot
// sequence and the arithmetic per element are those of the unblocked
// elimination; only the order of the sums changes.
#pragma once
#include "rgf_device.cuh"

namespace rgf {

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

template <int NB>
struct StagedCfg {
  static constexpr int PM = NB < 64 ? NB : 64;   // output tile
  static constexpr int PN = PM;
  static constexpr int KC = 16;                  // K chunk
  static constexpr int LDS = PM + 2;             // shared pitch (complex values)
  static constexpr int WARPS_M = 4, WARPS_N = 2;
  static constexpr int WM = PM / WARPS_M, WN = PN / WARPS_N;   // warp tile
  static constexpr int TM = WM / 8, TN = WN / 8;               // 8x8 subtiles per warp
  static constexpr int STAGE = 2 * KC * LDS;                   // complex values per stage (A + B)
  static constexpr int PW = NB >= 256 ? 16 : 32;               // inverse panel width
  static constexpr bool SMEM_INV = NB <= 64;                   // whole inverse in shared memory
  static constexpr size_t GEMM_SMEM = size_t(2) * STAGE * sizeof(double2);
  static constexpr size_t INV_SMEM = SMEM_INV ? size_t(NB) * NB * sizeof(double2)
                                              : size_t(NB) * PW * sizeof(double2);
  static constexpr size_t SMEM = GEMM_SMEM > INV_SMEM ? GEMM_SMEM : INV_SMEM;
  static_assert(TM >= 1 && TN >= 1, "tile");
  static_assert(PM % (8 * WARPS_M) == 0 && PN % (8 * WARPS_N) == 0, "tile");
};

// C = op(A) op(B); epi(i, j, v) once per element by its owner thread.
// M, N multiples of PM; K multiple of KC.  Caller synchronises afterwards.
template <int NB, class Epi>
__device__ __forceinline__ void gemm_staged(int M, int N, int K, const double2* A, int lda, bool cA,
                                            const double2* B, int ldb, bool cB, double2* stage,
                                            Epi&& epi) {
  using C = StagedCfg<NB>;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wm = (warp % C::WARPS_M) * C::WM, wn = (warp / C::WARPS_M) * C::WN;
  const double a_sg = cA ? -1.0 : 1.0, b_sg = cB ? -1.0 : 1.0;
  const int nchunks = K / C::KC;
  for (int tm0 = 0; tm0 < M; tm0 += C::PM) {
    for (int tn0 = 0; tn0 < N; tn0 += C::PN) {
      auto load_chunk = [&](int kc, int s) {
        double2* As = stage + s * C::STAGE;
        double2* Bs = As + C::KC * C::LDS;
        const int k0 = kc * C::KC;
        // op(A)[m][k] -> As[k*LDS + m]
        for (int e = tid; e < C::PM * C::KC; e += kThreads) {
          int m, k;
          if (!cA) { m = e % C::PM; k = e / C::PM; } else { k = e % C::KC; m = e / C::KC; }
          const double2* src = cA ? A + (size_t)(k0 + k) + (size_t)(tm0 + m) * lda
                                  : A + (size_t)(tm0 + m) + (size_t)(k0 + k) * lda;
          cp_async16(As + k * C::LDS + m, src);
        }
        // op(B)[k][n] -> Bs[k*LDS + n]
        for (int e = tid; e < C::PN * C::KC; e += kThreads) {
          int n, k;
          if (cB) { n = e % C::PN; k = e / C::PN; } else { k = e % C::KC; n = e / C::KC; }
          const double2* src = cB ? B + (size_t)(tn0 + n) + (size_t)(k0 + k) * ldb
                                  : B + (size_t)(k0 + k) + (size_t)(tn0 + n) * ldb;
          cp_async16(Bs + k * C::LDS + n, src);
        }
        cp_async_commit();
      };
      double cr[C::TM][C::TN][2], ci[C::TM][C::TN][2];
#pragma unroll
      for (int a = 0; a < C::TM; a++)
#pragma unroll
        for (int b = 0; b < C::TN; b++) cr[a][b][0] = cr[a][b][1] = ci[a][b][0] = ci[a][b][1] = 0.0;
      load_chunk(0, 0);
      for (int kc = 0; kc < nchunks; kc++) {
        if (kc + 1 < nchunks) {
          load_chunk(kc + 1, (kc + 1) & 1);
          cp_async_wait<1>();
        } else {
          cp_async_wait<0>();
        }
        __syncthreads();
        const double2* As = stage + (kc & 1) * C::STAGE;
        const double2* Bs = As + C::KC * C::LDS;
#pragma unroll
        for (int k4 = 0; k4 < C::KC; k4 += 4) {
          double2 av[C::TM], bv[C::TN];
#pragma unroll
          for (int a = 0; a < C::TM; a++) av[a] = As[(k4 + t) * C::LDS + wm + 8 * a + g];
#pragma unroll
          for (int b = 0; b < C::TN; b++) bv[b] = Bs[(k4 + t) * C::LDS + wn + 8 * b + g];
#pragma unroll
          for (int a = 0; a < C::TM; a++) {
            const double ar = av[a].x, ai = av[a].y * a_sg;
#pragma unroll
            for (int b = 0; b < C::TN; b++) {
              const double br = bv[b].x, bi = bv[b].y * b_sg;
              dmma884(cr[a][b][0], cr[a][b][1], ar, br);
              dmma884(cr[a][b][0], cr[a][b][1], -ai, bi);
              dmma884(ci[a][b][0], ci[a][b][1], ar, bi);
              dmma884(ci[a][b][0], ci[a][b][1], ai, br);
            }
          }
        }
        __syncthreads();  // the stage is refilled by the next iteration
      }
#pragma unroll
      for (int a = 0; a < C::TM; a++)
#pragma unroll
        for (int b = 0; b < C::TN; b++)
#pragma unroll
          for (int c = 0; c < 2; c++)
            epi(tm0 + wm + 8 * a + g, tn0 + wn + 8 * b + 2 * t + c,
                make_double2(cr[a][b][c], ci[a][b][c]));
    }
  }
}

// Blocked Gauss-Jordan inverse of the NB x NB block X (global memory, ld NB,
// overwritten), result into dst (and dst2).  Rt: a global scratch block for
// the panel rows R.  panel: shared memory of NB * PW complex values.
// Returns 1 (and zeros dst) on a zero pivot.
template <int NB>
__device__ int gj_invert_blocked(double2* X, double2* dst, double2* dst2, double2* Rt,
                                 double2* panel, double2* stage, SmemInv& s) {
  using C = StagedCfg<NB>;
  constexpr int PW = C::PW;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) s.singular = 0;
  for (int p0 = 0; p0 < NB; p0 += PW) {
    // (a) panel columns -> shared memory, column-major with ld NB
    for (int e = tid; e < NB * PW; e += kThreads) panel[e] = X[(size_t)p0 * NB + e];
    __syncthreads();
    // (b) unblocked elimination of the panel
    for (int c = 0; c < PW; c++) {
      const int k = p0 + c;
      double2* col = panel + (size_t)c * NB;
      if (warp == 0) {
        double best = -1.0;
        int bi = k;
        for (int i = k + lane; i < NB; i += 32) {
          const double v = cabs1(col[i]);
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
          s.pivval = col[bi];
          s.perm[k] = bi;
          if (best == 0.0) s.singular = 1;
        }
      }
      __syncthreads();
      if (s.singular) break;
      const int q = s.piv;
      const double2 pinv = crecip(s.pivval);
      for (int j = tid; j < PW; j += kThreads) {
        const double2 a = panel[k + (size_t)j * NB];
        const double2 b = panel[q + (size_t)j * NB];
        if (q != k) panel[q + (size_t)j * NB] = a;
        const double2 r = (j == c) ? pinv : cmul(b, pinv);
        panel[k + (size_t)j * NB] = r;
        s.rowk[j] = r;
      }
      __syncthreads();
      for (int i = tid; i < NB; i += kThreads) s.fcol[i] = (i == k) ? czero() : col[i];
      __syncthreads();
      for (int e = tid; e < NB * PW; e += kThreads) {
        const int j = e / NB, i = e - j * NB;
        if (i == k) continue;
        const double2 f = s.fcol[i];
        const double2 x = (j == c) ? czero() : panel[e];
        const double2 r = s.rowk[j];
        panel[e] = make_double2(x.x - (f.x * r.x - f.y * r.y), x.y - (f.x * r.y + f.y * r.x));
      }
      __syncthreads();
    }
    if (s.singular) break;
    // (c) panel back; (d) its row interchanges on the other columns
    for (int e = tid; e < NB * PW; e += kThreads) X[(size_t)p0 * NB + e] = panel[e];
    for (int j = tid; j < NB; j += kThreads) {
      if (j >= p0 && j < p0 + PW) continue;
      double2* colj = X + (size_t)j * NB;
      for (int c = 0; c < PW; c++) {
        const int k = p0 + c, q = s.perm[k];
        if (q != k) { const double2 tmp = colj[k]; colj[k] = colj[q]; colj[q] = tmp; }
      }
    }
    __syncthreads();
    // (e) R = X[P, :] (PW x NB, ld PW)
    for (int e = tid; e < NB * PW; e += kThreads) {
      const int j = e / PW, c = e - j * PW;
      Rt[e] = X[(p0 + c) + (size_t)j * NB];
    }
    __syncthreads();
    // (f) other columns: X[P,j] = U[P,:] R[:,j];  X[i,j] += U[i,:] R[:,j]
    gemm_staged<NB>(NB, NB, PW, X + (size_t)p0 * NB, NB, false, Rt, PW, false, stage,
                    [&](int i, int j, double2 v) {
                      if (j >= p0 && j < p0 + PW) return;
                      double2* x = X + i + (size_t)j * NB;
                      *x = (i >= p0 && i < p0 + PW) ? v : cadd(*x, v);
                    });
    __syncthreads();
  }
  const int sing = s.singular;
  if (sing) {
    for (int e = tid; e < NB * NB; e += kThreads) {
      dst[e] = czero();
      if (dst2) dst2[e] = czero();
    }
    __syncthreads();
    return 1;
  }
  if (tid == 0) {
    for (int j = 0; j < NB; j++) s.colsrc[j] = j;
    for (int k = NB - 1; k >= 0; k--) {
      const int q = s.perm[k];
      if (q != k) { const int tmp = s.colsrc[k]; s.colsrc[k] = s.colsrc[q]; s.colsrc[q] = tmp; }
    }
  }
  __syncthreads();
  for (int e = tid; e < NB * NB; e += kThreads) {
    const int j = e / NB, i = e - j * NB;
    const double2 v = X[i + (size_t)s.colsrc[j] * NB];
    dst[e] = v;
    if (dst2) dst2[e] = v;
  }
  __syncthreads();
  return 0;
}

}  // namespace rgf
