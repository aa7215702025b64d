// rgf_mixed.cu -- the persistent kernel of the mixed-precision form
// (RGF_PREC_MIXED, nb = 128) and the batched block operations
// (rgf_block_product / rgf_block_inverse) that expose its product and inverse.
//
// The mixed kernel runs the chain of green_RGF_RS (src/green_rgf.f90:
// 3950-4164) like the FP64 kernel, one (device, k, E) task per CTA at a
// time, with one CTA per SM (its split-integer operands fill most of the
// SM's shared memory): Sancho-Rubio (:4451-4537) and the lead self-energies
// in FP64 DMMA, every other block product as a split-integer product on
// tcgen05 and every other inverse as the refined FP32 inverse
// (rgf_mixed.cuh).  Each CTA allocates its TMEM once, keeps it for all its
// tasks and frees it before it returns, also after a bounded wait gave up.
#include <algorithm>
#include <cstdio>

#include "rgf_internal.h"
#include "rgf_mixed.cuh"
#include "rgf_solver.cuh"

namespace rgf {

namespace {

// Extra scratch blocks of a mixed-form slot beyond slot_elems_for(): the
// refined inverse Y, the residual R and the product staging block.
constexpr int kMixedExtraBlocks = 3;

struct MixedCta {
  uint32_t tmem;
  MixState st;
};

// The dynamic shared memory of a mixed-form CTA, rounded up to a 1024-byte
// boundary of the shared window: the tensor cores read the digit operands
// through matrix descriptors whose start addresses must be aligned (an
// operand 80 bytes past a 128-byte boundary was read three 16-byte rows
// late), and the runtime places dynamic shared memory after the static
// variables at only a 16-byte boundary (0xcd0 here).  The array is declared
// with 16-byte alignment so that the compiler cannot fold the rounding
// away; the launch reserves 1024 bytes of slack for it.
__device__ __forceinline__ unsigned char* aligned_dyn(unsigned char* p) {
  const uint32_t s = mx::smem_u32(p);
  return p + ((1024u - (s & 1023u)) & 1023u);
}

// Shared set-up of a mixed-form CTA: the two mbarriers and the TMEM
// allocation (warp 0).
__device__ __forceinline__ void mixed_cta_begin(unsigned char* dyn, uint32_t* tmem_slot, MixedCta& c) {
  const int warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) {
    mx::mbar_init(mx::smem_u32(dyn + mx::BAR_OFF));        // level buffer 0
    mx::mbar_init(mx::smem_u32(dyn + mx::BAR_OFF + 8));    // level buffer 1
    mx::mbar_init(mx::smem_u32(dyn + mx::BAR_OFF + 16));   // drain after a failed wait
  }
  if (warp == 0) {
    mx::tmem_alloc(tmem_slot, mx::TMEM_COLS);
    __syncwarp();
  }
  mx::fence_before_sync();
  __syncthreads();
  mx::fence_after_sync();
  c.tmem = *tmem_slot;
  c.st.ph0 = c.st.ph1 = 0;
  c.st.ok = 1;
  c.st.pad = 0;
}

// Frees the TMEM.  A CTA whose wait gave up first waits (bounded again) for
// the MMAs it may still have in flight: a commit to the third, never used
// mbarrier completes its first phase once every MMA issued before it is done.
__device__ __forceinline__ void mixed_cta_end(unsigned char* dyn, MixedCta& c) {
  if (!c.st.ok && threadIdx.x == 0) {
    mx::mma_commit(mx::smem_u32(dyn + mx::BAR_OFF + 16));
    mx::mbar_wait(mx::smem_u32(dyn + mx::BAR_OFF + 16), 0u);
  }
  mx::fence_before_sync();
  __syncthreads();
  mx::fence_after_sync();
  if ((threadIdx.x >> 5) == 0) mx::tmem_dealloc(c.tmem, mx::TMEM_COLS);
}

__device__ __noinline__ void task_mixed128(const KParams& p, int64_t t, double2* slot, Smem& sm,
                                           unsigned char* dyn, MixedCta& c) {
  DInfo* info = p.info ? p.info + t : nullptr;
  const DDev dv = p.devs[p.tasks[t].dev];
  const size_t n2 = 128 * 128;
  double2* temps = slot + 2 * (size_t)dv.nx * n2;
  MixedOps ops(sm.inv, sm.red, dyn, temps + (size_t)T_INV * n2, temps + (size_t)T_RT * n2,
               temps + (size_t)kNumTemps * n2, temps + (size_t)(kNumTemps + 1) * n2,
               temps + (size_t)(kNumTemps + 2) * n2, c.tmem, c.st);
  Solver<MixedOps> s(p.o, dv.nx, sm, ops, slot, 128, (int)dv.nx);
  s.run(p.tasks[t], dv, info, p.progress ? p.progress + t : nullptr);
  if (info && threadIdx.x == 0) {
    info->n_inv += ops.n_fallback + ops.n_fp64_inv;
    info->pad = ops.n_pairs;
    if (ops.n_fallback) info->status |= RGF_ST_REFINE_NC;
    if (!c.st.ok) info->status |= RGF_ST_TIMEOUT;
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kThreads, 1) rgf_mixed_kernel(KParams p) {
  extern __shared__ __align__(16) unsigned char dyn_raw[];
  __shared__ Smem sm;
  __shared__ uint32_t tmem_slot;
  unsigned char* dyn_smem = aligned_dyn(dyn_raw);
  MixedCta c;
  mixed_cta_begin(dyn_smem, &tmem_slot, c);
  double2* slot = p.work + (size_t)blockIdx.x * p.slot_elems;
  for (;;) {
    if (threadIdx.x == 0) sm.task = atomicAdd(p.queue, 1);
    __syncthreads();
    const int64_t q = sm.task;
    __syncthreads();
    if (q >= p.n_tasks) break;
    const int64_t t = p.order ? p.order[q] : q;
    const DDev& dv = p.devs[p.tasks[t].dev];
    if (dv.nm != 128 || dv.nx < 2 || dv.Sii ||
        slot_elems_for(128, dv.nx) + kMixedExtraBlocks * 128 * 128 > p.slot_elems) {
      if (p.info && threadIdx.x == 0) p.info[t].status = RGF_ST_BAD_TASK;
      continue;
    }
    task_mixed128(p, t, slot, sm, dyn_smem, c);
    if (!c.st.ok) break;
  }
  mixed_cta_end(dyn_smem, c);
}

// ------------------------------------------------------------------ blocks
// One CTA per block (grid-stride): mode 0 product op(A) op(B) split-integer
// with ns slices, 1 product FP64 (nb = 128), 2 inverse refined, 3 inverse
// FP64.  ws: 5 global blocks per CTA (X, X1, Y, R, product staging).
template <int NB>
__device__ void block_fp64_inverse(const double2* A, double2* C, double2* ws, Smem& sm, unsigned char* dyn,
                                   int32_t* status, int b) {
  StagedOps<NB> ops(sm.inv, (double2*)dyn, ws, ws + NB * NB, NB);
  for (int e = threadIdx.x; e < NB * NB; e += kThreads) ops.X[e] = A[e];
  __syncthreads();
  const int sing = ops.invert(NB, C, nullptr);
  if (threadIdx.x == 0 && status) status[b] = sing ? RGF_ST_SINGULAR : 0;
  __syncthreads();
}

template <int NB>
__global__ void __launch_bounds__(kThreads, 1) rgf_block_fp64_inv_kernel(const double2* X, double2* Xi,
                                                                         int64_t count, double2* ws,
                                                                         int32_t* status) {
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  __shared__ Smem sm;
  double2* w = ws + (size_t)blockIdx.x * 4 * NB * NB;
  for (int64_t b = blockIdx.x; b < count; b += gridDim.x)
    block_fp64_inverse<NB>(X + (size_t)b * NB * NB, Xi + (size_t)b * NB * NB, w, sm, dyn_smem, status, (int)b);
}

__global__ void __launch_bounds__(kThreads, 1) rgf_block_mixed_kernel(int mode, int ns, const double2* A, int cA,
                                                                      const double2* B, int cB, double2* C,
                                                                      int64_t count, double2* ws,
                                                                      int32_t* status) {
  extern __shared__ __align__(16) unsigned char dyn_raw[];
  __shared__ Smem sm;
  __shared__ uint32_t tmem_slot;
  unsigned char* dyn_smem = aligned_dyn(dyn_raw);
  MixedCta c;
  mixed_cta_begin(dyn_smem, &tmem_slot, c);
  constexpr size_t n2 = 128 * 128;
  double2* w = ws + (size_t)blockIdx.x * 5 * n2;
  MixedOps ops(sm.inv, sm.red, dyn_smem, w, w + n2, w + 2 * n2, w + 3 * n2, w + 4 * n2, c.tmem, c.st);
  for (int64_t b = blockIdx.x; b < count && c.st.ok; b += gridDim.x) {
    const double2* a = A + (size_t)b * n2;
    double2* o = C + (size_t)b * n2;
    if (mode == 0 || mode == 1) {
      const double2* bb = B + (size_t)b * n2;
      auto epi = [&](int i, int j, double2 v) { o[i + (size_t)j * 128] = v; };
      if (mode == 0) ops.gemm_mixed(a, cA != 0, bb, cB != 0, epi, ns > 0 ? ns : mx::S);
      else ops.f64.gemm(128, a, cA != 0, bb, cB != 0, epi);
      __syncthreads();
      if (threadIdx.x == 0 && status) status[b] = c.st.ok ? 0 : RGF_ST_TIMEOUT;
    } else {
      for (int e = threadIdx.x; e < (int)n2; e += kThreads) ops.X[e] = a[e];
      __syncthreads();
      ops.n_fallback = 0;
      const int sing = mode == 2 ? ops.invert_mixed(o, nullptr) : ops.f64.invert(128, o, nullptr);
      if (threadIdx.x == 0 && status)
        status[b] = (sing ? RGF_ST_SINGULAR : 0) | (ops.n_fallback ? RGF_ST_REFINE_NC : 0) |
                    (c.st.ok ? 0 : RGF_ST_TIMEOUT);
      __syncthreads();
    }
  }
  mixed_cta_end(dyn_smem, c);
}

}  // namespace

size_t mixed_smem() { return (size_t)mx::SMEM_BYTES + 1024; }
int64_t mixed_slot_elems(int64_t nx) { return slot_elems_for(128, nx) + kMixedExtraBlocks * 128 * 128; }

cudaError_t launch_mixed(const KParams& p, int grid, cudaStream_t st, bool set_attr) {
  const size_t smem = mixed_smem();
  if (set_attr) {
    cudaError_t e = cudaFuncSetAttribute(rgf_mixed_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  rgf_mixed_kernel<<<grid, kThreads, smem, st>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_block_mixed(int mode, int ns, const double2* A, int cA, const double2* B, int cB, double2* C,
                               int64_t count, double2* ws, int grid, int32_t* status, cudaStream_t st) {
  const size_t smem = mixed_smem();
  cudaError_t e = cudaFuncSetAttribute(rgf_block_mixed_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  rgf_block_mixed_kernel<<<grid, kThreads, smem, st>>>(mode, ns, A, cA, B, cB, C, count, ws, status);
  return cudaGetLastError();
}

cudaError_t launch_block_fp64_inv(int nb, const double2* X, double2* Xi, int64_t count, double2* ws, int grid,
                                  int32_t* status, cudaStream_t st) {
  cudaError_t e = cudaSuccess;
  switch (nb) {
    case 32: {
      const size_t smem = StagedCfg<32>::SMEM;
      e = cudaFuncSetAttribute(rgf_block_fp64_inv_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e == cudaSuccess) rgf_block_fp64_inv_kernel<32><<<grid, kThreads, smem, st>>>(X, Xi, count, ws, status);
      break;
    }
    case 64: {
      const size_t smem = StagedCfg<64>::SMEM;
      e = cudaFuncSetAttribute(rgf_block_fp64_inv_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e == cudaSuccess) rgf_block_fp64_inv_kernel<64><<<grid, kThreads, smem, st>>>(X, Xi, count, ws, status);
      break;
    }
    case 128: {
      const size_t smem = StagedCfg<128>::SMEM;
      e = cudaFuncSetAttribute(rgf_block_fp64_inv_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e == cudaSuccess) rgf_block_fp64_inv_kernel<128><<<grid, kThreads, smem, st>>>(X, Xi, count, ws, status);
      break;
    }
    default:
      return cudaErrorInvalidValue;
  }
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}

}  // namespace rgf
