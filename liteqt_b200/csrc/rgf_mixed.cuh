// rgf_mixed.cuh -- the mixed-precision block operations of RGF_PREC_MIXED
// (nb = 128) on the sm_100a tensor cores.
//
// Product C = op(A) op(B) of two complex FP64 128 x 128 blocks, split-integer
// (Ozaki scheme I) on tcgen05.mma.kind::i8:
//   * every row r of op(A) is scaled by a power of two 2^(P - E_r), with
//     2^E_r > max_k |op(A)[r][k]| (real and imaginary parts), and rounded to
//     a P-bit integer, P = 8 S - 2 = 46; every column j of op(B) likewise;
//   * each integer is written as S = 6 balanced base-256 digits in
//     [-128, 127] (slice p = 0 the most significant): adding
//     0x80 * sum_b 256^b to the integer makes its bytes the digits plus 128;
//   * the digit products sum_k a_p[r][k] b_q[k][j] are exact in int32 (at
//     most S K 2^14 in magnitude), accumulated in tensor memory (TMEM) by the
//     MMA; the pairs with p + q = L share one accumulator ("level" L) --
//     one MMA multiplies slice p with all B slices q at once, into columns
//     offset so that (p, q) lands on level p + q -- and the pairs with
//     p + q >= S are dropped (weights 2^-8S and below of the leading pair);
//   * the levels are combined in FP64 registers and scaled back:
//     C[r][j] = 2^(E_r + F_j - 12) sum_L T_L 2^(-8 L).
// The complex product runs as two real MMAs per A slice and K step,
// a_re x [b_re | b_im]_q and a_im x [b_re | b_im]_q over the B slices q, into
// two accumulators, combined on the way out: Re = ArBr - AiBi,
// Im = ArBi + AiBr.  Error per element: below about
// 2^-(8S-4) n max_k |op(A)[r][k]| max_k |op(B)[k][j]| (rounding of both
// operands to P bits of their row / column maxima, and the dropped pairs).
//
// Shared memory: the digits of op(A) for all K stay resident (S x 2 x 16 KB);
// the digits of op(B) for one tile of NT = 16 output columns
// (S x 2 NT x 128 B) are rewritten per tile, the next tile's FP64 values
// already in flight in registers while the current tile's MMAs run.  Both
// use a K-major layout without swizzle whose 8-row x 16-byte core matrices
// are adjacent along the rows (SBO = 128 B) and whole K groups of 16 apart
// (LBO = 16 x rows): element (r, k) of an R-row operand at
// (k / 16) 16 R + 16 r + k % 16.  A K group of all rows is one contiguous
// run, so the tensor cores' operand reads and the digit stores (consecutive
// rows from consecutive threads) do not collide in the shared-memory banks,
// which they do when 8-row groups sit 1 KB apart.  The B slices of a tile
// are consecutive row groups of one operand.  Operand bases are 1024-byte
// aligned.  TMEM holds every level of a tile (2 S x 2 NT columns); the MMAs
// are issued in two groups with a commit each, so the CTA reads the first
// levels back (tcgen05.ld) and accumulates them in FP64 while the tensor
// cores run the second group.
//
// Inverse: Gauss-Jordan with partial pivoting in FP32, the matrix in
// registers (64 complex values per thread), then Newton-Schulz steps
// Y <- Y + Y (I - X Y) with the residual I - X Y formed by the split-integer
// product against the FP64 matrix X, until n max|I - X Y| <= 2^-21 before the
// last step (so the step leaves it near 2^-42).  A zero FP32 pivot or a
// residual that does not fall below 1/2 sends the block to the FP64
// Gauss-Jordan inverse of the plain form (status RGF_ST_REFINE_NC).
//
// Every wait on an mbarrier is bounded (about one second of clock64); a wait
// that gives up marks the CTA failed, skips the remaining block operations of
// its task and makes the kernel return after freeing its TMEM.
#pragma once
#include <cstdint>

#include "rgf_device.cuh"
#include "rgf_solver.cuh"
#include "rgf_staged.cuh"

namespace rgf {
namespace mx {

constexpr int NB = 128;               // block size of the mixed form
constexpr int S = 6;                  // digit slices per operand
constexpr int P = 8 * S - 2;          // fixed-point bits of the scaled integers
constexpr int NT = 16;                // output columns per tile
constexpr int NTILE = NB / NT;
constexpr int KSTEPS = NB / 32;       // MMA K steps (32 int8 each)
constexpr uint32_t A_BLK = NB * NB;                 // bytes of one (slice, component) of op(A)
constexpr uint32_t A_BYTES = S * 2 * A_BLK;         // all digits of op(A)
constexpr uint32_t B_SL = 2 * NT;                   // B tile rows of one slice: real parts, imaginary
constexpr uint32_t B_ROWS = S * B_SL;               // all slices, as one operand (slice q at rows q B_SL ..)
constexpr uint32_t B_BYTES = B_ROWS * NB;
constexpr uint32_t EXP_OFF = A_BYTES + B_BYTES;     // int rowexp[NB], colexp[NB]
constexpr uint32_t BAR_OFF = EXP_OFF + 2 * NB * 4;  // 3 mbarriers
constexpr uint32_t SMEM_BYTES = BAR_OFF + 64;
constexpr uint32_t D_I = S * B_SL;                  // TMEM: levels x [ArBr | ArBi], then levels x [AiBr | AiBi]
constexpr int H1_SLICES = (S + 1) / 2;              // A slices of the first MMA group (levels 0 .. H1-1 final)
constexpr uint32_t TMEM_COLS = 512;
static_assert(2 * D_I <= TMEM_COLS, "every level of a tile in TMEM");
static_assert(B_ROWS <= 256, "one MMA spans every B slice (N <= 256)");
static_assert(TMEM_COLS == 32 || TMEM_COLS == 64 || TMEM_COLS == 128 || TMEM_COLS == 256 ||
              TMEM_COLS == 512, "TMEM allocation is a power of two >= 32 columns");
static_assert(SMEM_BYTES + 1024 <= 227 * 1024, "one CTA per SM, with 1 KB of alignment slack");
static_assert(StagedCfg<NB>::SMEM <= A_BYTES, "the FP64 operations alias the digit area");
static_assert(NT == 16, "the drain reads 8 columns per thread of each 16-column block");
// instruction descriptor: D s32 (bits 4-5 = 2), A and B s8 (bits 7-9, 10-12
// = 1), both K-major, M = 128 (bits 24-28: M >> 4); N in bits 17-22 (N >> 3)
constexpr uint32_t IDESC_BASE = (2u << 4) | (1u << 7) | (1u << 10) | (((uint32_t)NB >> 4) << 24);
__host__ __device__ constexpr uint32_t idesc_n(uint32_t n) { return IDESC_BASE | ((n >> 3) << 17); }
constexpr long long kWaitCycles = 2000000000ll;     // ~1 s at the B200 boost clock

// ------------------------------------------------------------------ PTX
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
// Shared-memory matrix descriptor, SWIZZLE_NONE K-major: start >> 4 in bits
// 0-13, LBO >> 4 (byte distance of the two 16-byte K halves of an MMA's
// K = 32) in 16-29, SBO >> 4 (byte distance of consecutive 8-row groups) in
// 32-45, version 1 in bits 46-47.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
__device__ __forceinline__ void mma_i8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}
// One lane of a converged warp (elect.sync): the lane that issues the MMAs
// and commits while its whole warp computes the (warp-uniform) descriptors.
__device__ __forceinline__ bool elect_one() {
  uint32_t pred = 0;
  asm volatile("{\n\t.reg .pred P1;\n\telect.sync _|P1, 0xffffffff;\n\tselp.b32 %0, 1, 0, P1;\n\t}\n"
               : "=r"(pred));
  return pred != 0;
}
__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_init(uint32_t mbar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Bounded wait for the completion of phase `parity` of an mbarrier.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  const long long t0 = clock64();
  for (;;) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (ok) return true;
    if (clock64() - t0 > kWaitCycles) return false;
  }
}
// 32 lanes x 8 consecutive 32-bit columns of TMEM -> 8 registers.
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, int32_t (&v)[8]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                 "=r"(v[7])
               : "r"(taddr));
}
// Completes the outstanding tcgen05.ld of this thread; the registers are
// passed through so no use of them is scheduled before the wait.
__device__ __forceinline__ void tmem_wait_ld(int32_t (&a)[8], int32_t (&b)[8], int32_t (&c)[8], int32_t (&d)[8]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]),
                 "+r"(b[0]), "+r"(b[1]), "+r"(b[2]), "+r"(b[3]), "+r"(b[4]), "+r"(b[5]), "+r"(b[6]), "+r"(b[7]),
                 "+r"(c[0]), "+r"(c[1]), "+r"(c[2]), "+r"(c[3]), "+r"(c[4]), "+r"(c[5]), "+r"(c[6]), "+r"(c[7]),
                 "+r"(d[0]), "+r"(d[1]), "+r"(d[2]), "+r"(d[3]), "+r"(d[4]), "+r"(d[5]), "+r"(d[6]), "+r"(d[7])::"memory");
}
// TMEM allocation by warp 0 (all its lanes, converged: the .sync.aligned
// forms need the whole warp at the same instruction); the address lands in
// *dst.
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  __syncwarp();
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  __syncwarp();
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// ------------------------------------------------------------------ split
// Biased exponent of max(|re|, |im|) (0 for zero and subnormal values).
__device__ __forceinline__ unsigned bexp(double2 v) {
  const unsigned a = (unsigned)(((unsigned long long)__double_as_longlong(v.x) >> 52) & 0x7FF);
  const unsigned b = (unsigned)(((unsigned long long)__double_as_longlong(v.y) >> 52) & 0x7FF);
  return a > b ? a : b;
}
// 2^(P - E) for a row whose largest entry has biased exponent X (E = X - 1022),
// as a double; 0 for rows below 2^-(1022 - P + 36) (treated as zero) and
// for Inf / NaN rows (their results are made NaN by the output scale).
__device__ __forceinline__ double row_scale(unsigned X) {
  const int be = 1023 + P - ((int)X - 1022);
  if (X == 0 || X >= 2047 || be < 1 || be > 2046) return 0.0;
  return __longlong_as_double((long long)be << 52);
}
// 0x80 in each of the S low bytes: added to a P-bit integer it makes every
// byte its balanced digit plus 128.
constexpr unsigned long long kBias = ((1ull << (8 * S)) - 1) / 255ull * 0x80ull;
// Balanced digits (as bytes d + 128) of round(x * scale): the bytes of
// round(x * scale) + kBias.  The rounding is the magic-number form:
// fma(x, scale, 1.5 * 2^52) rounds the exact product to an integer in the
// low mantissa bits (|x * scale| <= 2^P < 2^51).
__device__ __forceinline__ unsigned long long digits_of(double x, double scale) {
  const double r = fma(x, scale, 6755399441055744.0);
  return (unsigned long long)__double_as_longlong(r) + (kBias - 0x4338000000000000ull);
}
// Byte b of y[4q .. 4q+3], packed low to high, as signed digits (^ 0x80).
template <int N>
__device__ __forceinline__ uint32_t gather_byte(const unsigned long long (&y)[N], int q, int b) {
  const uint32_t s = (uint32_t)(b & 3) | ((uint32_t)((b & 3) + 4) << 4);
  uint32_t w0, w1, w2, w3;
  if (b < 4) {
    w0 = (uint32_t)y[4 * q]; w1 = (uint32_t)y[4 * q + 1]; w2 = (uint32_t)y[4 * q + 2]; w3 = (uint32_t)y[4 * q + 3];
  } else {
    w0 = (uint32_t)(y[4 * q] >> 32); w1 = (uint32_t)(y[4 * q + 1] >> 32);
    w2 = (uint32_t)(y[4 * q + 2] >> 32); w3 = (uint32_t)(y[4 * q + 3] >> 32);
  }
  const uint32_t lo = __byte_perm(w0, w1, s);
  const uint32_t hi = __byte_perm(w2, w3, s);
  return __byte_perm(lo, hi, 0x5410) ^ 0x80808080u;
}
// Writes the S digit slices of 16 (8) consecutive K values of one operand
// row (one component): slice p (0 = most significant) goes to
// base + p * stride.
__device__ __forceinline__ void store_digits16(const unsigned long long (&y)[16], unsigned char* base,
                                               uint32_t stride) {
#pragma unroll
  for (int p = 0; p < S; p++) {
    const int b = S - 1 - p;
    uint4 w;
    w.x = gather_byte(y, 0, b);
    w.y = gather_byte(y, 1, b);
    w.z = gather_byte(y, 2, b);
    w.w = gather_byte(y, 3, b);
    *reinterpret_cast<uint4*>(base + (size_t)p * stride) = w;
  }
}
__device__ __forceinline__ void store_digits8(const unsigned long long (&y)[8], unsigned char* base,
                                              uint32_t stride) {
#pragma unroll
  for (int p = 0; p < S; p++) {
    const int b = S - 1 - p;
    uint2 w;
    w.x = gather_byte(y, 0, b);
    w.y = gather_byte(y, 1, b);
    *reinterpret_cast<uint2*>(base + (size_t)p * stride) = w;
  }
}
// Offset of the 16-byte row segment (row r, K group g) of an operand of
// `rows` rows.
__device__ __forceinline__ uint32_t kmaj_off(int r, int g, int rows) {
  return (uint32_t)(g * 16 * rows + 16 * r);
}

// op(M)[r][k0 + kk] for kk < N (row-operand view: element (r, k) of op(M) is
// M[r + k n] for op N, conj(M[k + r n]) for op C) ...
template <int N>
__device__ __forceinline__ void load_row(const double2* M, bool c, int r, int k0, double2 (&v)[N]) {
  if (!c) {
#pragma unroll
    for (int kk = 0; kk < N; kk++) v[kk] = M[r + (size_t)(k0 + kk) * NB];
  } else {
#pragma unroll
    for (int kk = 0; kk < N; kk++) {
      const double2 x = M[(k0 + kk) + (size_t)r * NB];
      v[kk] = make_double2(x.x, -x.y);
    }
  }
}
// ... and op(M)[k0 + kk][j] (column-operand view: M[k + j n] for op N,
// conj(M[j + k n]) for op C).
template <int N>
__device__ __forceinline__ void load_col(const double2* M, bool c, int j, int k0, double2 (&v)[N]) {
  if (!c) {
#pragma unroll
    for (int kk = 0; kk < N; kk++) v[kk] = M[(k0 + kk) + (size_t)j * NB];
  } else {
#pragma unroll
    for (int kk = 0; kk < N; kk++) {
      const double2 x = M[j + (size_t)(k0 + kk) * NB];
      v[kk] = make_double2(x.x, -x.y);
    }
  }
}
// x 2^e for the output scale: a multiplication by a constructed power of
// two when 2^e is a normal double, scalbn otherwise.
__device__ __forceinline__ double scale2(double x, int e) {
  if (e > -1022 && e < 1024) return x * __longlong_as_double((long long)(e + 1023) << 52);
  return scalbn(x, e);
}

}  // namespace mx

// ------------------------------------------------------------------ policy
// State of a CTA's tensor-core pipeline that outlives a task: the parities of
// the two level-buffer mbarriers and the failure flag of the bounded waits.
struct MixState {
  uint32_t ph0, ph1;
  int ok;
  int pad;
};

// Block operations of the mixed form: the split-integer product and the
// refined FP32 inverse while `mixed_on`, the plain FP64 operations
// (StagedOps<128>) otherwise (Sancho-Rubio and its self-energies).
struct MixedOps {
  static constexpr bool kMixed = true;
  static constexpr int kMinBlocks = 1;
  StagedOps<128> f64;
  SmemInv& inv;
  SmemRed& red;
  unsigned char* sm;    // dynamic shared memory (1024-aligned)
  double2* X;           // the matrix to invert (global)
  double2* Y;           // refined inverse (global scratch block)
  double2* R;           // residual I - X Y (global scratch block)
  double2* Cs;          // product staging: the tiles' results, then one epilogue pass
  uint32_t tmem;        // TMEM base address of this CTA
  MixState& st;         // mbarrier parities, failure flag (the CTA's, across tasks)
  bool mixed_on = false;
  int n_pairs = 0;      // digit-pair products (4 real 128^3 int8 products each)
  int n_fallback = 0;   // refined inverses that fell back to FP64
  int n_fp64_inv = 0;   // inverses of the device chain run in FP64

  __device__ MixedOps(SmemInv& i, SmemRed& r, unsigned char* dyn, double2* slot_inv, double2* slot_rt,
                      double2* y, double2* res, double2* cs, uint32_t tm, MixState& s)
      : f64(i, (double2*)dyn, slot_inv, slot_rt, 128), inv(i), red(r), sm(dyn), X(slot_inv), Y(y), R(res),
        Cs(cs), tmem(tm), st(s) {}
  __device__ bool ok() const { return st.ok != 0; }

  __device__ double2* scratch() const { return (double2*)sm; }
  __device__ int* rowexp() const { return (int*)(sm + mx::EXP_OFF); }
  __device__ int* colexp() const { return (int*)(sm + mx::EXP_OFF) + mx::NB; }
  __device__ uint32_t bar(int b) const { return mx::smem_u32(sm + mx::BAR_OFF + 8 * b); }

  // bounded wait on level buffer b; the CTA agrees on the outcome
  __device__ void wait_buf(int b) {
    uint32_t& ph = b ? st.ph1 : st.ph0;
    const bool w = mx::mbar_wait(bar(b), ph);
    ph ^= 1u;
    st.ok = __syncthreads_and(w && st.ok) ? 1 : 0;
  }

  // Row exponents of op(A) and column exponents of op(B) (biased, of the
  // largest real or imaginary part).  Raw element idx of an operand is
  // (i, j) = (idx % n, idx / n); its row in op(A) is j for op C, i for op N,
  // its column in op(B) is i for op C, j for op N.  Loads go out 16 at a
  // time per thread.
  __device__ void exponents(const double2* A, bool cA, const double2* B, bool cB) {
    int* rx = rowexp();
    int* cx = colexp();
    const int tid = threadIdx.x;
    if (tid < mx::NB) { rx[tid] = 0; cx[tid] = 0; }
    __syncthreads();
    constexpr int PER = (mx::NB * mx::NB) / kThreads;   // 64 elements a thread
    constexpr int BATCH = 32;
#pragma unroll 1
    for (int which = 0; which < 2; which++) {
      const double2* M = which ? B : A;
      // key = idx % n when (A, op N) or (B, op C), else idx / n
      const bool mod_key = which ? cB : !cA;
      int* dst = which ? cx : rx;
      unsigned local = 0;
      unsigned wmax[PER / 32] = {};
#pragma unroll
      for (int m0 = 0; m0 < PER; m0 += BATCH) {
        unsigned e[BATCH];
#pragma unroll
        for (int b = 0; b < BATCH; b++) e[b] = mx::bexp(M[tid + (m0 + b) * kThreads]);
        if (mod_key) {
#pragma unroll
          for (int b = 0; b < BATCH; b++) local = e[b] > local ? e[b] : local;
        } else {
          // key (tid + m kThreads) >> 7 = tid / 128 + 2 m is warp-uniform: the
          // warp's maximum for element m is kept by lane m % 32 (two per lane)
#pragma unroll
          for (int b = 0; b < BATCH; b++) {
            const unsigned w = __reduce_max_sync(0xffffffffu, e[b]);
            if (((m0 + b) & 31) == (tid & 31)) wmax[(m0 + b) >> 5] = w;
          }
        }
      }
      if (mod_key) {
        atomicMax(dst + (tid & (mx::NB - 1)), (int)local);
      } else {
#pragma unroll
        for (int u = 0; u < PER / 32; u++)
          atomicMax(dst + ((tid >> 7) + 2 * ((tid & 31) + 32 * u)), (int)wmax[u]);
      }
    }
    __syncthreads();
  }

  // Digits of op(A) (all K) into shared memory: thread tid takes row
  // tid % 128 and the K groups g = tid / 128 + 2 i; consecutive threads write
  // consecutive rows (16 bytes apart).
  __device__ void split_a(const double2* A, bool cA) {
    const int tid = threadIdx.x;
    const int r = tid & (mx::NB - 1);
    const double sc = mx::row_scale((unsigned)rowexp()[r]);
#pragma unroll 1
    for (int g = tid >> 7; g < mx::NB / 16; g += kThreads / mx::NB) {
      double2 v[16];
      mx::load_row<16>(A, cA, r, 16 * g, v);
      unsigned long long y[16];
      const uint32_t off = mx::kmaj_off(r, g, mx::NB);
#pragma unroll
      for (int kk = 0; kk < 16; kk++) y[kk] = mx::digits_of(v[kk].x, sc);
      mx::store_digits16(y, sm + off, 2 * mx::A_BLK);
#pragma unroll
      for (int kk = 0; kk < 16; kk++) y[kk] = mx::digits_of(v[kk].y, sc);
      mx::store_digits16(y, sm + mx::A_BLK + off, 2 * mx::A_BLK);
    }
  }

  // The B tile of columns j0 .. j0 + NT: thread tid takes column
  // j = (tid >> 1) % NT, K group g = tid / (2 NT) and half tid & 1 of its 16
  // K values.  load_b fetches the thread's 8 values of op(B) (issued before
  // the previous tile's MMAs are waited for, so the loads overlap them),
  // store_b writes their digits: row j (real parts) and NT + j (imaginary
  // parts) of each slice.
  __device__ void load_b(const double2* B, bool cB, int j0, double2 (&v)[8]) const {
    const int tid = threadIdx.x;
    const int j = (tid >> 1) % mx::NT, g = tid / (2 * mx::NT), hk = tid & 1;
    mx::load_col<8>(B, cB, j0 + j, 16 * g + 8 * hk, v);
  }
  __device__ void store_b(int j0, const double2 (&v)[8]) {
    const int tid = threadIdx.x;
    const int j = (tid >> 1) % mx::NT, g = tid / (2 * mx::NT), hk = tid & 1;
    const double sc = mx::row_scale((unsigned)colexp()[j0 + j]);
    unsigned char* base = sm + mx::A_BYTES + 8 * hk;
    unsigned long long y[8];
#pragma unroll
    for (int kk = 0; kk < 8; kk++) y[kk] = mx::digits_of(v[kk].x, sc);
    mx::store_digits8(y, base + mx::kmaj_off(j, g, mx::B_ROWS), 16 * mx::B_SL);
#pragma unroll
    for (int kk = 0; kk < 8; kk++) y[kk] = mx::digits_of(v[kk].y, sc);
    mx::store_digits8(y, base + mx::kmaj_off(mx::NT + j, g, mx::B_ROWS), 16 * mx::B_SL);
  }
  static_assert(2 * mx::NT * (mx::NB / 16) == kThreads, "one B half-group per thread");

  // The MMAs of A slices p0 .. p1-1, then a commit to mbarrier b.  One MMA
  // multiplies slice p of op(A) (real or imaginary digits) with every B slice
  // q < ns - p at once (N = (ns - p) x 2 NT: the slices are consecutive row
  // groups of the B operand) into TMEM columns starting p x 2 NT further
  // along, so the product of slices p and q lands on level p + q's columns:
  // the levels accumulate without a separate pass per digit pair, in S MMAs
  // per component and K step instead of S (S + 1) / 2.  Slice 0, K step 0
  // writes every level (accumulate off); all others accumulate, so the MMAs
  // of a tile are issued by one thread, in order.  Called by every lane of
  // one warp: the descriptors are warp-uniform values and one elected lane
  // issues (a single diverged thread issued each MMA in ~100 cycles).  A
  // descriptor's start address sits in its low bits (addresses < 256 KB, no
  // carry), so an operand offset is added to the base descriptor as
  // offset >> 4.
  __device__ void issue_slices(int p0, int p1, int ns, int b) {
    const uint32_t sa = mx::smem_u32(sm), sb = sa + mx::A_BYTES;
    constexpr uint32_t la = 16 * mx::NB, lb = 16 * mx::B_ROWS;        // K-group strides
    const uint64_t dA0 = mx::sdesc(sa, la, 128);
    const uint64_t dB0 = mx::sdesc(sb, lb, 128);
    const bool leader = mx::elect_one();
    mx::fence_after_sync();
    for (int p = p0; p < p1; p++) {
      const uint32_t idesc = mx::idesc_n((uint32_t)(ns - p) * mx::B_SL);
      const uint32_t d_r = tmem + (uint32_t)p * mx::B_SL;              // levels x [ArBr | ArBi]
      const uint32_t d_i = d_r + mx::D_I;                              // levels x [AiBr | AiBi]
      const uint64_t ar = dA0 + ((uint64_t)(2 * p) * mx::A_BLK >> 4);
      const uint64_t ai = ar + (mx::A_BLK >> 4);
#pragma unroll
      for (int ks = 0; ks < mx::KSTEPS; ks++) {
        // an MMA's K = 32 is K groups 2 ks and 2 ks + 1
        const uint32_t acc = (p > 0 || ks > 0) ? 1u : 0u;
        if (leader) {
          mx::mma_i8(d_r, ar + (2 * ks * la >> 4), dB0 + (2 * ks * lb >> 4), idesc, acc);
          mx::mma_i8(d_i, ai + (2 * ks * la >> 4), dB0 + (2 * ks * lb >> 4), idesc, acc);
        }
      }
    }
    if (leader) mx::mma_commit(bar(b));
    __syncwarp();
  }

  // Adds levels L0 .. L1-1 of the thread's 8 output columns (TMEM lane r,
  // columns 8 h ..) to re / im in FP64: Re = ArBr - AiBi, Im = ArBi + AiBr,
  // level L weighted 2^-8L.
  __device__ void drain_levels(int L0, int L1, uint32_t tl, int h, double (&re)[8], double (&im)[8]) {
    mx::fence_after_sync();
    __syncwarp();   // tcgen05.ld is warp-collective (.sync.aligned)
    for (int L = L0; L < L1; L++) {
      const uint32_t cb = tl + (uint32_t)L * mx::B_SL + 8 * h;
      int32_t rbr[8], rbi[8], ibr[8], ibi[8];
      mx::tmem_ld8(cb, rbr);                           // ArBr
      mx::tmem_ld8(cb + mx::NT, rbi);                  // ArBi
      mx::tmem_ld8(cb + mx::D_I, ibr);                 // AiBr
      mx::tmem_ld8(cb + mx::D_I + mx::NT, ibi);        // AiBi
      mx::tmem_wait_ld(rbr, rbi, ibr, ibi);
      const double w = __longlong_as_double((long long)(1023 - 8 * L) << 52);   // 2^-8L
#pragma unroll
      for (int c = 0; c < 8; c++) {
        re[c] = fma((double)(rbr[c] - ibi[c]), w, re[c]);
        im[c] = fma((double)(rbi[c] + ibr[c]), w, im[c]);
      }
    }
    mx::fence_before_sync();
  }

  // C = op(A) op(B) by the split-integer product with ns <= S slices;
  // epi(i, j, v) once per element by the thread that owns it.  A must not be
  // written by epi (op(A) is read once, before the first epilogue); B is
  // read tile by tile.
  //
  // Per tile of 16 output columns the MMAs go out in two groups with a
  // commit each: A slices 0 .. h1-1, after which levels 0 .. h1-1 are final
  // and the CTA reads them back while the tensor cores run the second group;
  // then the remaining levels.  The next tile's B digits are written once
  // every MMA of the tile has completed, its MMAs issued, and the finished
  // tile's outputs scaled and stored while they run.
  template <class Epi>
  __device__ void gemm_mixed(const double2* A, bool cA, const double2* B, bool cB, Epi&& epi, int ns = mx::S) {
    if (!ok()) return;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int h1 = ns < mx::H1_SLICES ? ns : mx::H1_SLICES;
    const bool two = h1 < ns;
    exponents(A, cA, B, cB);
    double2 bv[8];
    load_b(B, cB, 0, bv);
    split_a(A, cA);
    store_b(0, bv);
    mx::fence_async_smem();
    __syncthreads();
    if (mx::NTILE > 1) load_b(B, cB, mx::NT, bv);          // tile 1's values, in flight
    if (warp == 0) {
      issue_slices(0, h1, ns, 0);
      if (two) issue_slices(h1, ns, ns, 1);
    }
    const int r = 32 * (warp & 3) + lane;                  // output row (TMEM lane)
    const int h = warp >> 2;                               // which 8 of the tile's 16 columns
    const uint32_t tl = tmem + ((uint32_t)(32 * (warp & 3)) << 16);
    const int xr = rowexp()[r];
    for (int tile = 0; tile < mx::NTILE; tile++) {
      const int j0 = tile * mx::NT;
      double re[8], im[8];
#pragma unroll
      for (int c = 0; c < 8; c++) re[c] = im[c] = 0.0;
      wait_buf(0);                                         // levels 0 .. h1-1 final
      if (!ok()) return;
      drain_levels(0, h1, tl, h, re, im);
      if (two) {
        wait_buf(1);                                       // every MMA of the tile done
        if (!ok()) return;
        drain_levels(h1, ns, tl, h, re, im);
      }
      __syncthreads();                                     // TMEM read by all; B tile free
      if (tile + 1 < mx::NTILE) {
        store_b(j0 + mx::NT, bv);
        mx::fence_async_smem();
        __syncthreads();
        if (warp == 0) {
          issue_slices(0, h1, ns, 0);
          if (two) issue_slices(h1, ns, ns, 1);
        }
        if (tile + 2 < mx::NTILE) load_b(B, cB, j0 + 2 * mx::NT, bv);
      }
#pragma unroll
      for (int c = 0; c < 8; c++) {
        const int j = j0 + 8 * h + c;
        const int yc = colexp()[j];
        double2 v;
        if (xr >= 2047 || yc >= 2047) {
          v = make_double2(__longlong_as_double(0x7ff8000000000000ll), __longlong_as_double(0x7ff8000000000000ll));
        } else {
          const int e = xr + yc - 2056;        // 2^(E_r + F_j - 12), E = X - 1022
          v = make_double2(mx::scale2(re[c], e), mx::scale2(im[c], e));
        }
        Cs[r + (size_t)j * mx::NB] = v;
      }
    }
    __syncthreads();
    // One elementwise pass of the epilogue over the staged product, eight
    // elements a thread at a time: the epilogues' own global loads (H, Gl,
    // ...) go out together instead of eight per tile behind each drain.
    for (int base = tid; base < mx::NB * mx::NB; base += 8 * kThreads) {
      double2 v[8];
#pragma unroll
      for (int u = 0; u < 8; u++) v[u] = Cs[base + u * kThreads];
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const int idx = base + u * kThreads;
        epi(idx & (mx::NB - 1), idx >> 7, v[u]);
      }
    }
    n_pairs += ns * (ns + 1) / 2;
  }

  template <class Epi>
  __device__ void gemm(int n, const double2* A, bool cA, const double2* B, bool cB, Epi&& epi) {
    if (mixed_on) {
      gemm_mixed(A, cA, B, cB, epi);
      __syncthreads();   // the next operation may overwrite the digit area
    } else {
      f64.gemm(n, A, cA, B, cB, epi);
    }
  }

  // ---------------------------------------------------------------- inverse
  __device__ double block_max(double v) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (lane == 0) red.v[warp] = v;
    __syncthreads();
    double m = 0.0;
#pragma unroll
    for (int w = 0; w < kWarps; w++) m = fmax(m, red.v[w]);
    __syncthreads();
    return m;
  }

  // FP32 Gauss-Jordan inverse of X (FP64, global) with the matrix in
  // registers: thread tid owns row tid % 128 and the 64 consecutive columns
  // of half tid / 128; per column a pivot search by warp reductions (largest
  // |re| + |im|, first row on ties), the scaled pivot row and row k published
  // in shared memory, two barriers.  Writes the inverse (as FP64) to Y in
  // its column order.  Returns 1 on a zero pivot.
  __device__ __noinline__ int gj_f32() {
    constexpr int N = mx::NB, CPT = N * N / kThreads, WPC = N / 32;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int i = tid % N, hh = tid / N, j0 = hh * CPT;
    float2* fraw = (float2*)sm;              // [2][N]
    float2* rr = fraw + 2 * N;               // [2][N]
    float2* rk = rr + 2 * N;                 // [2][N]
    float2* pinvw = rk + 2 * N;              // [2][WPC]
    unsigned* pk = (unsigned*)(pinvw + 2 * WPC);
    int* pi = (int*)(pk + 2 * WPC);
    float2 x[CPT];
#pragma unroll
    for (int m = 0; m < CPT; m++) {
      const double2 v = X[i + (size_t)(j0 + m) * N];
      x[m] = make_float2((float)v.x, (float)v.y);
    }
    if (tid == 0) inv.singular = 0;
    __syncthreads();
    for (int k = 0; k < N; k++) {
      const int par = k & 1, hc = k / CPT, mc = k - hc * CPT;   // k, hc, mc uniform
      if (hh == hc) {
        float2 v = x[0];
#pragma unroll
        for (int m = 1; m < CPT; m++)
          if (m == mc) v = x[m];
        fraw[par * N + i] = v;
        const float av = fabsf(v.x) + fabsf(v.y);
        unsigned key = 0u;
        if (i >= k) key = !(av == av) ? 1u : (av == 0.0f ? 2u : __float_as_uint(av) + 2u);
        const float sv = fmaxf(fabsf(v.x), fabsf(v.y));
        float2 pv = make_float2(0.f, 0.f);
        if (sv > 0.0f) {
          const float ar = v.x / sv, ai = v.y / sv;
          const float d = 1.0f / ((ar * ar + ai * ai) * sv);
          pv = make_float2(ar * d, -ai * d);
        }
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
        if (key <= 2u) inv.singular = 1;
        inv.perm[k] = (int16_t)q;
      }
      if (i == q) {
        const float2 pinv = pinvw[par * WPC + wq];
#pragma unroll
        for (int m = 0; m < CPT; m++) {
          const float2 a = x[m];
          rr[par * N + j0 + m] = (j0 + m == k) ? pinv
                                               : make_float2(a.x * pinv.x - a.y * pinv.y, a.x * pinv.y + a.y * pinv.x);
        }
      }
      if (i == k) {
#pragma unroll
        for (int m = 0; m < CPT; m++) rk[par * N + j0 + m] = x[m];
      }
      __syncthreads();
      if (i == k) {
#pragma unroll
        for (int m = 0; m < CPT; m++) x[m] = rr[par * N + j0 + m];
      } else {
        const float2 f = (i == q) ? rk[par * N + k] : fraw[par * N + i];
        if (i == q) {
#pragma unroll
          for (int m = 0; m < CPT; m++) x[m] = rk[par * N + j0 + m];
        }
        if (hh == hc) {
#pragma unroll
          for (int m = 0; m < CPT; m++)
            if (m == mc) x[m] = make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int m = 0; m < CPT; m++) {
          const float2 rj = rr[par * N + j0 + m];
          x[m] = make_float2(x[m].x - (f.x * rj.x - f.y * rj.y), x[m].y - (f.x * rj.y + f.y * rj.x));
        }
      }
    }
    __syncthreads();
    if (inv.singular) return 1;
    if (tid == 0) {
      for (int j = 0; j < N; j++) inv.colsrc[j] = (int16_t)j;
      for (int k = N - 1; k >= 0; k--) {
        const int q = inv.perm[k];
        if (q != k) { const int16_t t = inv.colsrc[k]; inv.colsrc[k] = inv.colsrc[q]; inv.colsrc[q] = t; }
      }
    }
    __syncthreads();
    for (int j = tid; j < N; j += kThreads) inv.coldst[inv.colsrc[j]] = (int16_t)j;
    __syncthreads();
#pragma unroll
    for (int m = 0; m < CPT; m++) Y[i + (size_t)inv.coldst[j0 + m] * N] = make_double2((double)x[m].x, (double)x[m].y);
    __syncthreads();
    return 0;
  }

  // Refined inverse of X into dst (and dst2).  Returns 1 on a singular
  // block (from the FP64 fallback, which zeroes dst as the reference does).
  __device__ int invert_mixed(double2* dst, double2* dst2) {
    constexpr int N = mx::NB;
    bool fine = ok() && gj_f32() == 0;
    for (int step = 0; fine && step < 4; step++) {
      double rmax = 0.0;
      gemm_mixed(X, false, Y, false, [&](int i, int j, double2 v) {   // R = I - X Y
        const double2 rv = make_double2((i == j ? 1.0 : 0.0) - v.x, -v.y);
        R[i + (size_t)j * N] = rv;
        rmax = fmax(rmax, fmax(fabs(rv.x), fabs(rv.y)));
      });
      __syncthreads();
      const double eps = (double)N * block_max(rmax);
      if (!ok() || !(eps < 0.5)) { fine = false; break; }
      const bool last = eps <= 4.76837158203125e-07;                    // 2^-21
      if (!last && step == 3) { fine = false; break; }
      gemm_mixed(Y, false, R, false, [&](int i, int j, double2 v) {    // Y += Y R
        const size_t idx = i + (size_t)j * N;
        const double2 y = cadd(Y[idx], v);
        Y[idx] = y;
        if (last) {
          dst[idx] = y;
          if (dst2) dst2[idx] = y;
        }
      });
      __syncthreads();
      if (last) return 0;
    }
    // FP64 Gauss-Jordan of the plain form (X is intact: the FP32 elimination
    // and the residual products only read it)
    n_fallback++;
    return f64.invert(N, dst, dst2);
  }

  // The chain's inverses: the FP64 Gauss-Jordan of the plain form.  The
  // refined FP32 inverse (invert_mixed) is correct but, with one CTA per SM,
  // slower than it (1.55 M cycles against 0.60 M at nb = 128: the FP32
  // elimination's column loop is latency-bound like the FP64 one, and the
  // residual products come on top), so it serves rgf_block_inverse only.
  __device__ int invert(int n, double2* dst, double2* dst2) {
    if (mixed_on) n_fp64_inv++;
    return f64.invert(n, dst, dst2);
  }
};

}  // namespace rgf
