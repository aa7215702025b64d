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
#include <type_traits>

#include "rgf_device.cuh"

namespace rgf {
// Internal linkage: every translation unit compiles its own copies, under its
// own register budget (the FP64 kernel's units cap at 128 registers, the
// mixed form's unit does not), so no out-of-line instance is shared.
namespace {

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
  static constexpr int NSTAGE = 3;                             // cp.async pipeline depth (>= 2)
  static constexpr int PW = NB >= 256 ? 16 : (NB >= 128 ? 48 : 32);  // inverse panel width (max)
  static constexpr bool SMEM_INV = NB <= 64;                   // whole inverse in shared memory
  // column pitch of the blocked inverse's shared panel (complex values): NB + 2
  // makes the rank-8 updates' fragment reads of 4 columns x 2 rows hit 8
  // distinct 16-byte bank groups (pitch NB: 4-way conflicts)
  static constexpr int LDP = SMEM_INV ? NB : NB + 2;
  static constexpr size_t GEMM_SMEM = size_t(NSTAGE) * STAGE * sizeof(double2);
  // inverse: the matrix (nb <= 64) or one panel, then the row / column vectors
  static constexpr size_t INV_MAT = SMEM_INV ? size_t(NB) * NB : size_t(LDP) * PW;
  // inverse scratch after the matrix / panel, per form (complex values):
  // blocked (nb >= 128): pivot row + multiplier column + 8 pivot rows of the
  // panel's other columns, which also covers the sub-block elimination's
  // scratch; register form (nb = 32); one-panel blocked form (nb = 64):
  // 8 pivot rows of the other columns, or the sub-block scratch
  static constexpr size_t SCR_SUB = 2 * size_t(NB) + 48 + size_t(NB) / 16;
  static constexpr size_t SCR_PANEL = 2 * size_t(NB) + 8 * size_t(PW);
  static constexpr size_t SCR_BLOCKED = SCR_PANEL > SCR_SUB ? SCR_PANEL : SCR_SUB;
  static constexpr size_t SCR_REG = 6 * size_t(NB) + size_t(NB) / 8 + 8;
  static constexpr size_t SCR_ONE = 8 * (size_t(NB) - 8) > SCR_SUB ? 8 * (size_t(NB) - 8) : SCR_SUB;
  static constexpr size_t INV_SCR = !SMEM_INV ? SCR_BLOCKED : (NB == 32 ? SCR_REG : SCR_ONE);
  static constexpr size_t INV_SMEM = (INV_MAT + INV_SCR) * sizeof(double2);
  static constexpr size_t SMEM = GEMM_SMEM > INV_SMEM ? GEMM_SMEM : INV_SMEM;
  // two CTAs per SM: 2 x (dynamic + static shared memory + 1 KB reserved)
  // within the SM's 228 KB
  static_assert(SMEM <= 108 * 1024 + 512, "shared memory for two CTAs per SM");
  static_assert(TM >= 1 && TN >= 1, "tile");
  static_assert(PM % (8 * WARPS_M) == 0 && PN % (8 * WARPS_N) == 0, "tile");
};

struct NoInit {};

// C = C0 + op(A) op(B); epi(i, j, v) once per element by its owner thread.
// C0 = init(i, j) when an init functor is given (read before the K loop, so
// its loads overlap the first chunks' copies), else 0.  M, N multiples of PM;
// K multiple of KC.  Caller synchronises afterwards.
template <int NB, class Init, class Epi>
__device__ __forceinline__ void gemm_staged_init(int M, int N, int K, const double2* A, int lda, bool cA,
                                                 const double2* B, int ldb, bool cB, double2* stage,
                                                 Init&& init, Epi&& epi, const int16_t* brow) {
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
      if constexpr (!std::is_same_v<std::decay_t<Init>, NoInit>) {
#pragma unroll
        for (int a = 0; a < C::TM; a++)
#pragma unroll
          for (int b = 0; b < C::TN; b++)
#pragma unroll
            for (int c = 0; c < 2; c++) {
              const double2 v = init(tm0 + wm + 8 * a + g, tn0 + wn + 8 * b + 2 * t + c);
              cr[a][b][c] = v.x;
              ci[a][b][c] = v.y;
            }
      }
      // prologue: chunks 0 .. NSTAGE-2 in flight; one commit group per chunk
      // (possibly empty), so at iteration kc "all but the newest NSTAGE-2
      // groups done" means chunk kc has landed.  One barrier per chunk: it
      // makes chunk kc visible and proves every warp done with chunk kc-1,
      // whose stage the refill after it reuses; the barrier before the
      // prologue frees the stages of the previous tile (or the caller's use
      // of the same shared memory).
      __syncthreads();
#pragma unroll
      for (int c = 0; c < C::NSTAGE - 1; c++) {
        if (c < nchunks) load_chunk(c, c);
        cp_async_commit();
      }
      for (int kc = 0; kc < nchunks; kc++) {
        cp_async_wait<C::NSTAGE - 2>();
        __syncthreads();
        if (kc + C::NSTAGE - 1 < nchunks) load_chunk(kc + C::NSTAGE - 1, (kc + C::NSTAGE - 1) % C::NSTAGE);
        cp_async_commit();
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
      }
      // every warp is done with the stages before any epilogue runs: an
      // epilogue may write shared memory the stages alias (the nb <= 64
      // inverse assembles its matrix there)
      __syncthreads();
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

template <int NB, class Epi>
__device__ __forceinline__ void gemm_staged(int M, int N, int K, const double2* A, int lda, bool cA,
                                            const double2* B, int ldb, bool cB, double2* stage,
                                            Epi&& epi, const int16_t* brow = nullptr) {
  gemm_staged_init<NB>(M, N, K, A, lda, cA, B, ldb, cB, stage, NoInit{}, epi, brow);
}

// Gauss-Jordan inverse (partial pivoting) of the N x N block X (shared
// memory; used for N = 32) with the matrix held in registers: thread tid owns row
// tid % N and the CPT = N^2 / 256 consecutive columns of group tid / N.  Per
// column k:
//   (1) the owners of column k publish it and reduce the pivot key per warp
//       (redux.sync), each forming the reciprocal of its entry meanwhile;
//       barrier;
//   (2) every thread combines the partials (largest key, first row on ties);
//       the owners of row q publish the scaled pivot row r_j = x_qj / x_qk,
//       the owners of row k publish row k; barrier;
//   (3) every thread updates its elements, x_ij - f_i r_j (column k: -f_i r_k).
// Key, tie and zero-pivot rules as gj_subblock.  At the end each thread
// writes its elements to dst (and dst2) in the inverse's column order
// (column c of the eliminated matrix is column coldst[c] of the inverse).
// scr: 6 N + 4 N/32 + 8 complex values of shared scratch, double-buffered by
// column parity.  Returns 1 (and zeros dst) on a zero pivot.
template <int N>
__device__ __noinline__ int gj_invert_reg(const double2* X, double2* dst, double2* dst2, SmemInv& s,
                                          double2* scr) {
  constexpr int CPT = N * N / kThreads;  // columns per thread
  constexpr int WPC = N / 32;            // warps owning one column
  static_assert(CPT * kThreads == N * N && N % 32 == 0 && CPT >= 1, "register inverse layout");
  const int tid = threadIdx.x, warp = tid >> 5;
  const int i = tid % N, h = tid / N, j0 = h * CPT;
  double2* fraw = scr;               // [2][N] column k before the step
  double2* rr = fraw + 2 * N;        // [2][N] scaled pivot row
  double2* rk = rr + 2 * N;          // [2][N] row k before the step
  double2* pinvw = rk + 2 * N;       // [2][WPC] winners' reciprocals
  unsigned* pk = reinterpret_cast<unsigned*>(pinvw + 2 * WPC);  // [2][WPC]
  int* pi = reinterpret_cast<int*>(pk + 2 * WPC);               // [2][WPC]
  double2 x[CPT];
#pragma unroll
  for (int m = 0; m < CPT; m++) x[m] = X[i + (j0 + m) * N];
  if (tid == 0) s.singular = 0;
  for (int k = 0; k < N; k++) {
    const int par = k & 1, hc = k / CPT, mc = k - hc * CPT;
    if (h == hc) {
      double2 v = x[0];
#pragma unroll
      for (int m = 1; m < CPT; m++)
        if (m == mc) v = x[m];
      fraw[par * N + i] = v;
      const double av = cabs1(v);
      unsigned key = 0u;
      if (i >= k) {
        const unsigned hi = (unsigned)((unsigned long long)__double_as_longlong(av) >> 32);
        key = !(av == av) ? 1u : (av == 0.0 ? 2u : (hi > 1u ? hi : 1u) + 2u);
      }
      const double2 pv = crecip(v);
      const unsigned kmax = __reduce_max_sync(0xffffffffu, key);
      const unsigned imin = __reduce_min_sync(0xffffffffu, key == kmax ? (unsigned)i : 0xffffffffu);
      if ((unsigned)i == imin) {
        const int w = warp - hc * WPC;
        pk[par * WPC + w] = kmax;
        pi[par * WPC + w] = i;
        pinvw[par * WPC + w] = pv;
      }
    }
    __syncthreads();
    unsigned key = pk[par * WPC];
    int q = pi[par * WPC], wq = 0;
#pragma unroll
    for (int w = 1; w < WPC; w++) {
      const unsigned ek = pk[par * WPC + w];
      const int ei = pi[par * WPC + w];
      if (ek > key || (ek == key && ei < q)) { key = ek; q = ei; wq = w; }
    }
    if (tid == 0) {
      if (key == 2u) s.singular = 1;
      s.perm[k] = (int16_t)q;
    }
    if (i == q) {
      const double2 pinv = pinvw[par * WPC + wq];
#pragma unroll
      for (int m = 0; m < CPT; m++) rr[par * N + j0 + m] = (j0 + m == k) ? pinv : cmul(x[m], pinv);
    }
    if (i == k) {
#pragma unroll
      for (int m = 0; m < CPT; m++) rk[par * N + j0 + m] = x[m];
    }
    __syncthreads();
    const double2 f = (i == k) ? czero() : (i == q ? rk[par * N + k] : fraw[par * N + i]);
#pragma unroll
    for (int m = 0; m < CPT; m++) {
      const int j = j0 + m;
      const double2 r = rr[par * N + j];
      if (i == k) {
        x[m] = r;
      } else {
        const double2 base = (i == q) ? rk[par * N + j] : x[m];
        const double2 xx = (j == k) ? czero() : base;
        x[m] = make_double2(xx.x - (f.x * r.x - f.y * r.y), xx.y - (f.x * r.y + f.y * r.x));
      }
    }
  }
  __syncthreads();
  if (s.singular) {
#pragma unroll
    for (int m = 0; m < CPT; m++) {
      dst[i + (j0 + m) * N] = czero();
      if (dst2) dst2[i + (j0 + m) * N] = czero();
    }
    __syncthreads();
    return 1;
  }
  if (tid == 0) {
    for (int j = 0; j < N; j++) s.colsrc[j] = (int16_t)j;
    for (int k = N - 1; k >= 0; k--) {
      const int q = s.perm[k];
      if (q != k) { const int16_t tmp = s.colsrc[k]; s.colsrc[k] = s.colsrc[q]; s.colsrc[q] = tmp; }
    }
  }
  __syncthreads();
  for (int j = tid; j < N; j += kThreads) s.coldst[s.colsrc[j]] = (int16_t)j;
  __syncthreads();
#pragma unroll
  for (int m = 0; m < CPT; m++) {
    const int o = i + s.coldst[j0 + m] * N;
    dst[o] = x[m];
    if (dst2) dst2[o] = x[m];
  }
  __syncthreads();
  return 0;
}

// Gauss-Jordan elimination of the KB = 8 panel columns sb0.. (pivot rows
// p0+sb0..) with the sub-block held in registers: thread tid owns row tid % NB
// and CPT consecutive columns of the sub-block.  Per column:
//   (1) the owners of the pivot column publish it and reduce the pivot key
//       per warp (redux.sync; partials to shared memory), each lane forming
//       the reciprocal of its own entry meanwhile so the winner's is ready;
//       barrier;
//   (2) every thread combines the partials (largest key, first row on ties);
//       the two owners of row q form the scaled pivot row r_j = x_qj / x_qc,
//       the owners of row k publish it, the panel's other columns get the
//       interchange; barrier;
//   (3) every thread updates its own elements, x_ij - f_i r_j.
// The pivot key is the high word of the bit pattern of |re|+|im| (monotonic
// for non-negative doubles), so entries within 2^-20 of each other count as
// equal and the first row among them is taken; rows above k have key 0, NaN
// entries key 1 (never chosen unless the whole column is NaN, then row k as
// the scalar search), exact zeros key 2 and every other entry a larger key.
// The per-element arithmetic is that of the unblocked elimination.  scr:
// 2 NB + 6 KB + 2 NB/32 complex values of scratch, double-buffered by column
// parity so one column's readers never race the next column's writers.
// Returns with the sub-block written back to the panel and a barrier passed;
// s.singular is set on a zero pivot.
template <int NB, int LD = NB>
__device__ __forceinline__ void gj_subblock(double2* panel, int PW, int p0, int sb0, double2* scr,
                                            int16_t* rmap, SmemInv& s) {
  constexpr int KB = 8;
  constexpr int CPT = KB * NB / kThreads;  // sub-block columns per thread
  constexpr int WPC = NB / 32;             // warps owning one column
  static_assert(CPT * kThreads == KB * NB && KB % CPT == 0, "sub-block layout");
  const int tid = threadIdx.x, warp = tid >> 5;
  const int i = tid % NB, h = tid / NB;
  double2* fraw = scr;           // [2][NB] the pivot column before the step
  double2* rr = scr + 2 * NB;    // [2][KB] the scaled pivot row r
  double2* rk = rr + 2 * KB;     // [2][KB] row k of the sub-block before the step
  double2* pinvw = rk + 2 * KB;  // [2][WPC] per-warp winner's reciprocal
  unsigned* pk = reinterpret_cast<unsigned*>(pinvw + 2 * WPC);  // [2][WPC] keys
  int* pi = reinterpret_cast<int*>(pk + 2 * WPC);               // [2][WPC] rows
  double2 x[CPT];
#pragma unroll
  for (int m = 0; m < CPT; m++) x[m] = panel[i + (size_t)(sb0 + h * CPT + m) * LD];
#pragma unroll
  for (int cc = 0; cc < KB; cc++) {
    const int k = p0 + sb0 + cc, par = cc & 1;
    const int hc = cc / CPT, mc = cc % CPT;
    if (h == hc) {
      const double2 v = x[mc];
      fraw[par * NB + i] = v;
      const double av = cabs1(v);
      unsigned key = 0u;
      if (i >= k) {
        const unsigned hi = (unsigned)((unsigned long long)__double_as_longlong(av) >> 32);
        key = !(av == av) ? 1u : (av == 0.0 ? 2u : (hi > 1u ? hi : 1u) + 2u);
      }
      const double2 pv = crecip(v);
      const unsigned kmax = __reduce_max_sync(0xffffffffu, key);
      const unsigned imin = __reduce_min_sync(0xffffffffu, key == kmax ? (unsigned)i : 0xffffffffu);
      if ((unsigned)i == imin) {
        const int w = warp - hc * WPC;
        pk[par * WPC + w] = kmax;
        pi[par * WPC + w] = i;
        pinvw[par * WPC + w] = pv;
      }
    }
    __syncthreads();
    unsigned key = pk[par * WPC];
    int q = pi[par * WPC], wq = 0;
#pragma unroll
    for (int w = 1; w < WPC; w++) {
      const unsigned ek = pk[par * WPC + w];
      const int ei = pi[par * WPC + w];
      if (ek > key || (ek == key && ei < q)) { key = ek; q = ei; wq = w; }
    }
    // largest |re|+|im| zero: flagged, and the caller discards the block
    if (key == 2u && tid == 0) s.singular = 1;
    if (tid == 0) {
      s.perm[k] = (int16_t)q;
      if (q != k) { const int16_t t = rmap[k]; rmap[k] = rmap[q]; rmap[q] = t; }
    }
    if (i == q) {
      const double2 pinv = pinvw[par * WPC + wq];
#pragma unroll
      for (int m = 0; m < CPT; m++) {
        const int jj = h * CPT + m;
        rr[par * KB + jj] = (jj == cc) ? pinv : cmul(x[m], pinv);
      }
    }
    if (i == k) {
#pragma unroll
      for (int m = 0; m < CPT; m++) rk[par * KB + h * CPT + m] = x[m];
    }
    if (q != k) {  // the panel's other columns: interchange rows k <-> q
      for (int j = tid; j < PW; j += kThreads) {
        if (j >= sb0 && j < sb0 + KB) continue;
        const double2 a = panel[k + (size_t)j * LD];
        panel[k + (size_t)j * LD] = panel[q + (size_t)j * LD];
        panel[q + (size_t)j * LD] = a;
      }
    }
    __syncthreads();
    const double2 f = (i == k) ? czero() : (i == q ? rk[par * KB + cc] : fraw[par * NB + i]);
#pragma unroll
    for (int m = 0; m < CPT; m++) {
      const int jj = h * CPT + m;
      const double2 r = rr[par * KB + jj];
      if (i == k) {
        x[m] = r;
      } else {
        const double2 base = (i == q) ? rk[par * KB + jj] : x[m];
        const double2 xx = (jj == cc) ? czero() : base;
        x[m] = make_double2(xx.x - (f.x * r.x - f.y * r.y), xx.y - (f.x * r.y + f.y * r.x));
      }
    }
  }
#pragma unroll
  for (int m = 0; m < CPT; m++) panel[i + (size_t)(sb0 + h * CPT + m) * LD] = x[m];
  __syncthreads();
}

// Rank-8 update of a panel's other columns after its sub-block sb0.. (pivot
// rows R = rows p0+sb0.. of those columns, before the update, gathered into
// rbuf, 8 x (PW - 8)):
//   X[i, j] = (i in sub-block rows ? 0 : X[i, j]) + sum_t U[i, t] R[t, j]
// on the FP64 tensor pipe: warp w owns rows 8 TMU w .. (TMU 8-row subtiles)
// and walks the 8-column subtiles of the other columns; K = 8 is two m8n8k4
// steps, U's fragments loaded once.  Ends with a barrier.
template <int NB, int LD = NB>
__device__ __forceinline__ void panel_rank8_update(double2* panel, int PW, int p0, int sb0, double2* rbuf) {
  constexpr int KB = 8;
  const int tid = threadIdx.x;
  const int nrest = PW - KB;
  if (nrest <= 0) return;
  for (int e = tid; e < KB * nrest; e += kThreads) {
    const int t = e % KB, jr = e / KB;
    const int j = jr < sb0 ? jr : jr + KB;
    rbuf[t + jr * KB] = panel[(p0 + sb0 + t) + (size_t)j * LD];
  }
  __syncthreads();
  constexpr int TMU = NB / (8 * (kThreads / 32));
  static_assert(TMU >= 1 && TMU * 8 * (kThreads / 32) == NB, "rows per warp");
  const int lane = tid & 31, warp = tid >> 5, g = lane >> 2, t4 = lane & 3;
  const int wm = warp * 8 * TMU;
  double2 av[2][TMU];
#pragma unroll
  for (int ks = 0; ks < 2; ks++)
#pragma unroll
    for (int a = 0; a < TMU; a++) av[ks][a] = panel[(wm + 8 * a + g) + (size_t)(sb0 + 4 * ks + t4) * LD];
  for (int b = 0; b < nrest / 8; b++) {
    double cr[TMU][1][2], ci[TMU][1][2];
#pragma unroll
    for (int a = 0; a < TMU; a++) cr[a][0][0] = cr[a][0][1] = ci[a][0][0] = ci[a][0][1] = 0.0;
#pragma unroll
    for (int ks = 0; ks < 2; ks++) {
      const double2 bv[1] = {rbuf[(4 * ks + t4) + (8 * b + g) * KB]};
      cmma_step<TMU, 1>(cr, ci, av[ks], bv, 1.0, 1.0);
    }
#pragma unroll
    for (int a = 0; a < TMU; a++)
#pragma unroll
      for (int c = 0; c < 2; c++) {
        const int i = wm + 8 * a + g, jr = 8 * b + 2 * t4 + c;
        const int j = jr < sb0 ? jr : jr + KB;
        const bool prow = i >= p0 + sb0 && i < p0 + sb0 + KB;
        const size_t o = i + (size_t)j * LD;
        const double2 x = prow ? czero() : panel[o];
        panel[o] = make_double2(x.x + cr[a][0][c], x.y + ci[a][0][c]);
      }
  }
  __syncthreads();
}

// Gauss-Jordan inverse (partial pivoting) of the NB x NB block X held whole
// in shared memory (NB = 64): the blocked form of gj_invert_blocked with one
// panel, i.e. 8-column sub-blocks eliminated with their elements in
// registers (gj_subblock) and the other columns updated by rank-8 DMMA
// products (panel_rank8_update); no trailing matrix.  Then dst[:, j] =
// X[:, colsrc[j]] undoes the interchanges (and dst2 the same).  scr: shared
// scratch of max(8 (NB - 8), 2 NB + 48 + NB / 16) complex values.  Returns 1
// (and zeros dst) on a zero pivot.
template <int NB>
__device__ __noinline__ int gj_invert_smem_blocked(double2* X, double2* dst, double2* dst2, SmemInv& s,
                                                   double2* scr) {
  constexpr int KB = 8;
  static_assert(NB % KB == 0, "whole sub-blocks");
  const int tid = threadIdx.x;
  if (tid == 0) s.singular = 0;
  for (int i = tid; i < NB; i += kThreads) s.rmap[i] = (int16_t)i;
  __syncthreads();
  for (int sb0 = 0; sb0 < NB; sb0 += KB) {
    gj_subblock<NB>(X, NB, 0, sb0, scr, s.rmap, s);
    if (s.singular) break;
    panel_rank8_update<NB>(X, NB, 0, sb0, scr);
  }
  if (s.singular) {
    for_each_elem(NB, [&](int, int, int idx) {
      dst[idx] = czero();
      if (dst2) dst2[idx] = czero();
    });
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
  for_each_elem(NB, [&](int i, int j, int idx) {
    const double2 v = X[i + s.colsrc[j] * NB];
    dst[idx] = v;
    if (dst2) dst2[idx] = v;
  });
  __syncthreads();
  return 0;
}

// Blocked Gauss-Jordan inverse of the NB x NB block X0 (global memory, ld
// NB, destroyed), result into dst (and dst2).  X1: a second global block.
// The row interchanges of a panel are never applied in place: the panel's
// update reads the permuted rows of the current matrix (row gather in the
// GEMM loader and in the accumulators' preload) and writes the next matrix,
// the two buffers alternating; the last panel writes dst itself, its columns
// in the inverse's order.  Dynamic shared memory: panel (NB x PW), pivot row
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
  double2* rowk = panel + (size_t)C::LDP * PWM;
  double2* fcol = rowk + PWM;
  int16_t* rmap = s.rmap;
  const int tid = threadIdx.x;
  double2* cur = X0;
  double2* nxt = X1;
  if (tid == 0) s.singular = 0;
  for (int p0 = 0; p0 < NB; p0 += PWM) {
    const int PW = (NB - p0) < PWM ? (NB - p0) : PWM;
    // (a) panel columns of the current matrix -> shared memory (pitch LDP)
    for (int e = tid; e < NB * PW; e += kThreads) {
      const int jj = e / NB, i = e - jj * NB;
      cp_async16(panel + i + (size_t)jj * C::LDP, cur + (size_t)p0 * NB + e);
    }
    cp_async_commit();
    for (int i = tid; i < NB; i += kThreads) rmap[i] = (int16_t)i;
    cp_async_wait<0>();
    __syncthreads();
    // (b) elimination of the panel in sub-blocks of KB columns: each sub-block
    //     is eliminated unblocked with its columns in registers (gj_subblock;
    //     its row interchanges applied to the whole panel), then the panel's
    //     other columns get the sub-block's
    //     transformation as one rank-KB update (the same U R form as the
    //     panel's own update below), so the panel is read and written once per
    //     sub-block instead of once per column.
    constexpr int KB = 8;
    static_assert(PWM % KB == 0 && (NB % PWM) % KB == 0, "panels of whole sub-blocks");
    double2* rbuf = fcol + NB;  // KB x PWM pivot rows of the other columns
    for (int sb0 = 0; sb0 < PW && !s.singular; sb0 += KB) {
      gj_subblock<NB, C::LDP>(panel, PW, p0, sb0, rowk, rmap, s);
      if (s.singular) break;
      panel_rank8_update<NB, C::LDP>(panel, PW, p0, sb0, rbuf);
    }
    if (s.singular) break;
    // the last panel writes the inverse itself: its column j is column
    // colsrc[j] of the eliminated matrix (the interchanges undone), i.e.
    // column c goes to coldst[c]
    const bool last = p0 + PW >= NB;
    if (last) {
      if (tid == 0) {
        for (int j = 0; j < NB; j++) s.colsrc[j] = (int16_t)j;
        for (int k = NB - 1; k >= 0; k--) {
          const int q = s.perm[k];
          if (q != k) { const int16_t tmp = s.colsrc[k]; s.colsrc[k] = s.colsrc[q]; s.colsrc[q] = tmp; }
        }
      }
      __syncthreads();
      for (int j = tid; j < NB; j += kThreads) s.coldst[s.colsrc[j]] = (int16_t)j;
      __syncthreads();
    }
    // (c) eliminated panel -> next matrix (its rows are already in the new order)
    for (int e = tid; e < NB * PW; e += kThreads) {
      const int jj = e / NB, i = e - jj * NB;
      const double2 v = panel[i + (size_t)jj * C::LDP];
      nxt[(size_t)p0 * NB + e] = v;
      if (last) {
        const size_t o = i + (size_t)s.coldst[p0 + jj] * NB;
        dst[o] = v;
        if (dst2) dst2[o] = v;
      }
    }
    __syncthreads();
    // (d) other columns: with R = rows rmap[P] of cur and U the panel,
    //     nxt[P, j] = U[P, :] R[:, j],   nxt[i, j] = cur[rmap[i], j] + U[i, :] R[:, j]
    gemm_staged_init<NB>(NB, NB, PW, nxt + (size_t)p0 * NB, NB, false, cur, NB, false, stage,
                         [&](int i, int j) {
                           const bool keep = (i < p0 || i >= p0 + PW) && (j < p0 || j >= p0 + PW);
                           return keep ? cur[(size_t)rmap[i] + (size_t)j * NB] : czero();
                         },
                         [&](int i, int j, double2 v) {
                           if (j >= p0 && j < p0 + PW) return;
                           if (last) {
                             const size_t o = i + (size_t)s.coldst[j] * NB;
                             dst[o] = v;
                             if (dst2) dst2[o] = v;
                           } else {
                             nxt[i + (size_t)j * NB] = v;
                           }
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
  return 0;
}

}  // namespace

}  // namespace rgf
