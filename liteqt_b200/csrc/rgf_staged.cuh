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
  static constexpr int NSTAGE = 3;                             // cp.async pipeline depth
  static constexpr int PW = NB >= 256 ? 16 : (NB >= 128 ? 48 : 32);  // inverse panel width (max)
  static constexpr bool SMEM_INV = NB <= 64;                   // whole inverse in shared memory
  static constexpr size_t GEMM_SMEM = size_t(NSTAGE) * STAGE * sizeof(double2);
  // inverse: the matrix (nb <= 64) or one panel, then the row / column vectors
  static constexpr size_t INV_MAT = SMEM_INV ? size_t(NB) * NB : size_t(NB) * PW;
  static constexpr size_t INV_SMEM = (INV_MAT + 2 * size_t(NB) + 8 * size_t(PW)) * sizeof(double2);
  static constexpr size_t SMEM = GEMM_SMEM > INV_SMEM ? GEMM_SMEM : INV_SMEM;
  static_assert(TM >= 1 && TN >= 1, "tile");
  static_assert(PM % (8 * WARPS_M) == 0 && PN % (8 * WARPS_N) == 0, "tile");
};

// C = op(A) op(B); epi(i, j, v) once per element by its owner thread.
// M, N multiples of PM; K multiple of KC.  Caller synchronises afterwards.
template <int NB, class Epi>
__device__ __forceinline__ void gemm_staged(int M, int N, int K, const double2* A, int lda, bool cA,
                                            const double2* B, int ldb, bool cB, double2* stage,
                                            Epi&& epi, const int16_t* brow = nullptr) {
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
          // brow: op(B) row k is row brow[k] of B (op N only)
          const int kr = brow ? (int)brow[k0 + k] : k0 + k;
          const double2* src = cB ? B + (size_t)(tn0 + n) + (size_t)(k0 + k) * ldb
                                  : B + (size_t)kr + (size_t)(tn0 + n) * ldb;
          cp_async16(Bs + k * C::LDS + n, src);
        }
      };
      double cr[C::TM][C::TN][2], ci[C::TM][C::TN][2];
#pragma unroll
      for (int a = 0; a < C::TM; a++)
#pragma unroll
        for (int b = 0; b < C::TN; b++) cr[a][b][0] = cr[a][b][1] = ci[a][b][0] = ci[a][b][1] = 0.0;
      // prologue: chunks 0 .. NSTAGE-2 in flight; one commit group per chunk
      // (possibly empty), so "all but the newest NSTAGE-1 groups done" means
      // chunk kc has landed
#pragma unroll
      for (int c = 0; c < C::NSTAGE - 1; c++) {
        if (c < nchunks) load_chunk(c, c);
        cp_async_commit();
      }
      for (int kc = 0; kc < nchunks; kc++) {
        if (kc + C::NSTAGE - 1 < nchunks) load_chunk(kc + C::NSTAGE - 1, (kc + C::NSTAGE - 1) % C::NSTAGE);
        cp_async_commit();
        cp_async_wait<C::NSTAGE - 1>();
        __syncthreads();
        const double2* As = stage + (kc % C::NSTAGE) * C::STAGE;
        const double2* Bs = As + C::KC * C::LDS;
#pragma unroll
        for (int k4 = 0; k4 < C::KC; k4 += 4) {
          double2 av[C::TM], bv[C::TN];
#pragma unroll
          for (int a = 0; a < C::TM; a++) av[a] = As[(k4 + t) * C::LDS + wm + 8 * a + g];
#pragma unroll
          for (int b = 0; b < C::TN; b++) bv[b] = Bs[(k4 + t) * C::LDS + wn + 8 * b + g];
          cmma_step<C::TM, C::TN>(cr, ci, av, bv, a_sg, b_sg);
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

// Blocked Gauss-Jordan inverse of the NB x NB block X0 (global memory, ld
// NB, destroyed), result into dst (and dst2).  X1: a second global block.
// The row interchanges of a panel are never applied in place: the panel's
// update reads the permuted rows of the current matrix (row gather in the
// GEMM loader and in the epilogue) and writes the next matrix, the two
// buffers alternating.  Dynamic shared memory: panel (NB x PW), pivot row
// (PW), multiplier column (NB) -- none of them is live during the update
// GEMM, which reuses the same memory as its staging buffers.  The panel's row
// map is read by that GEMM, so it lives in the static SmemInv.
// Returns 1 (and zeros dst) on a zero pivot.
template <int NB>
__device__ int gj_invert_blocked(double2* X0, double2* X1, double2* dst, double2* dst2,
                                 double2* smem, double2* stage, SmemInv& s) {
  using C = StagedCfg<NB>;
  constexpr int PWM = C::PW;
  double2* panel = smem;
  double2* rowk = panel + (size_t)NB * PWM;
  double2* fcol = rowk + PWM;
  int16_t* rmap = s.rmap;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double2* cur = X0;
  double2* nxt = X1;
  if (tid == 0) s.singular = 0;
  for (int p0 = 0; p0 < NB; p0 += PWM) {
    const int PW = (NB - p0) < PWM ? (NB - p0) : PWM;
    // (a) panel columns of the current matrix -> shared memory (ld NB)
    for (int e = tid; e < NB * PW; e += kThreads) panel[e] = cur[(size_t)p0 * NB + e];
    for (int i = tid; i < NB; i += kThreads) rmap[i] = (int16_t)i;
    __syncthreads();
    // (b) elimination of the panel in sub-blocks of KB columns: each sub-block
    //     is eliminated unblocked (its row interchanges applied to the whole
    //     panel at once), then the panel's other columns get the sub-block's
    //     transformation as one rank-KB update (the same U R form as the
    //     panel's own update below), so the panel is read and written once per
    //     sub-block instead of once per column.
    constexpr int KB = 8;
    double2* rbuf = fcol + NB;  // KB x PWM pivot rows of the other columns
    for (int sb0 = 0; sb0 < PW && !s.singular; sb0 += KB) {
      const int kb = (PW - sb0) < KB ? (PW - sb0) : KB;
      for (int c = sb0; c < sb0 + kb; c++) {
        const int k = p0 + c;
        const double2* col = panel + (size_t)c * NB;
        if (warp == 0) {  // pivot search
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
            s.akc = col[k];
            s.perm[k] = (int16_t)bi;
            if (best == 0.0) s.singular = 1;
            if (bi != k) { const int16_t t = rmap[k]; rmap[k] = rmap[bi]; rmap[bi] = t; }
          }
        }
        __syncthreads();
        if (s.singular) break;
        const int q = s.piv;
        const double2 pinv = crecip(s.pivval);
        // interchange rows k <-> q over the whole panel; scale row k in the
        // sub-block; multipliers f_i = old column entries
        for (int e = tid; e < PW + NB; e += kThreads) {
          if (e < PW) {
            const int j = e;
            const double2 a = panel[k + (size_t)j * NB];
            const double2 b = panel[q + (size_t)j * NB];
            if (q != k) panel[q + (size_t)j * NB] = a;
            if (j >= sb0 && j < sb0 + kb) {
              const double2 r = (j == c) ? pinv : cmul(b, pinv);
              panel[k + (size_t)j * NB] = r;
              rowk[j] = r;
            } else {
              panel[k + (size_t)j * NB] = b;
            }
          } else {
            const int i = e - PW;
            fcol[i] = (i == k) ? czero() : (i == q ? s.akc : col[i]);
          }
        }
        __syncthreads();
        for (int e = tid; e < NB * kb; e += kThreads) {
          const int jj = e / NB, i = e - jj * NB;
          const int j = sb0 + jj;
          if (i == k) continue;
          const double2 f = fcol[i];
          const size_t o = i + (size_t)j * NB;
          const double2 x = (j == c) ? czero() : panel[o];
          const double2 r = rowk[j];
          panel[o] = make_double2(x.x - (f.x * r.x - f.y * r.y), x.y - (f.x * r.y + f.y * r.x));
        }
        __syncthreads();
      }
      if (s.singular) break;
      // rank-kb update of the panel's other columns j (pivot rows R = rows
      // p0+sb0.. of those columns, before the update):
      //   X[i, j] = (i in sub-block rows ? 0 : X[i, j]) + sum_t U[i, t] R[t, j]
      const int nrest = PW - kb;
      if (nrest > 0) {
        for (int e = tid; e < kb * nrest; e += kThreads) {
          const int t = e % kb, jr = e / kb;
          const int j = jr < sb0 ? jr : jr + kb;
          rbuf[t + jr * KB] = panel[(p0 + sb0 + t) + (size_t)j * NB];
        }
        __syncthreads();
        // thread: one row i and a strided subset of the other columns
        constexpr int TPR = kThreads / NB > 0 ? kThreads / NB : 1;  // threads per row
        for (int i = tid % NB, part = tid / NB; i < NB && part < TPR; i += NB) {
          double2 u[KB];
#pragma unroll
          for (int t = 0; t < KB; t++) u[t] = t < kb ? panel[i + (size_t)(sb0 + t) * NB] : czero();
          const bool prow = i >= p0 + sb0 && i < p0 + sb0 + kb;
          for (int jr = part; jr < nrest; jr += TPR) {
            const int j = jr < sb0 ? jr : jr + kb;
            const size_t o = i + (size_t)j * NB;
            double2 x = prow ? czero() : panel[o];
#pragma unroll
            for (int t = 0; t < KB; t++) {
              if (t < kb) {
                const double2 r = rbuf[t + jr * KB];
                x.x += u[t].x * r.x - u[t].y * r.y;
                x.y += u[t].x * r.y + u[t].y * r.x;
              }
            }
            panel[o] = x;
          }
        }
        __syncthreads();
      }
    }
    if (s.singular) break;
    // (c) eliminated panel -> next matrix (its rows are already in the new order)
    for (int e = tid; e < NB * PW; e += kThreads) nxt[(size_t)p0 * NB + e] = panel[e];
    __syncthreads();
    // (d) other columns: with R = rows rmap[P] of cur and U the panel,
    //     nxt[P, j] = U[P, :] R[:, j],   nxt[i, j] = cur[rmap[i], j] + U[i, :] R[:, j]
    gemm_staged<NB>(NB, NB, PW, nxt + (size_t)p0 * NB, NB, false, cur, NB, false, stage,
                    [&](int i, int j, double2 v) {
                      if (j >= p0 && j < p0 + PW) return;
                      const size_t o = i + (size_t)j * NB;
                      nxt[o] = (i >= p0 && i < p0 + PW) ? v : cadd(cur[(size_t)rmap[i] + (size_t)j * NB], v);
                    },
                    rmap + p0);
    __syncthreads();
    double2* t = cur;
    cur = nxt;
    nxt = t;
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
    for (int j = 0; j < NB; j++) s.colsrc[j] = (int16_t)j;
    for (int k = NB - 1; k >= 0; k--) {
      const int q = s.perm[k];
      if (q != k) { const int16_t tmp = s.colsrc[k]; s.colsrc[k] = s.colsrc[q]; s.colsrc[q] = tmp; }
    }
  }
  __syncthreads();
  for (int e = tid; e < NB * NB; e += kThreads) {
    const int j = e / NB, i = e - j * NB;
    const double2 v = cur[i + (size_t)s.colsrc[j] * NB];
    dst[e] = v;
    if (dst2) dst2[e] = v;
  }
  __syncthreads();
  return 0;
}

}  // namespace rgf
