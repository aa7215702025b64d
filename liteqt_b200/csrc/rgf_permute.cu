// rgf_permute.cu -- the local transposes of the GW loop's energy <-> (i,j)
// redistribution (energies_to_ijs_2 / ijs_to_energies_2,
// src/green_rgf.f90:243-329): dst = RESHAPE(src, dst_shape, ORDER=order) of a
// complex(8) array, the Fortran intrinsic's meaning (src taken in array
// element order, dst filled with its subscripts running in the order
// order(1), order(2), ...), for pure transposes: dst_shape(order(k)) =
// src_shape(k).  HBM-bound data movement: 32 x 32 tiles through shared
// memory between the source's and the destination's contiguous dimensions
// (both sides coalesced), or contiguous runs when those coincide; index
// arithmetic once per tile, not per element.
#include <cstdint>
#include <cstdio>

#include <cuda_runtime.h>

#include "rgf_internal.h"

namespace {

constexpr int kMaxDims = 8;
constexpr int kTile = 32, kRows = 8;   // 32 x 32 tiles, 32 x 8 threads

// A pure transpose seen from the destination: its shape, the destination
// strides (column-major) and, per destination dimension, the stride of the
// source dimension feeding it.  db: the destination dimension fed by the
// source's innermost (stride-1) dimension.
struct PermPlan {
  int32_t nd, db;
  int64_t dshape[kMaxDims];
  int64_t sstr[kMaxDims];
  int64_t dstr[kMaxDims];
  int64_t tiles_a, tiles_b, batch;   // tiles along dimensions 0 and db, product of the others
};

// (source, destination) offsets of batch index r over every destination
// dimension except 0 and `skip`
__device__ __forceinline__ void batch_offsets(const PermPlan& p, int skip, int64_t r, int64_t& so, int64_t& dof) {
  so = 0;
  dof = 0;
  for (int d = 1; d < p.nd; d++) {
    if (d == skip) continue;
    const int64_t q = r % p.dshape[d];
    r /= p.dshape[d];
    so += q * p.sstr[d];
    dof += q * p.dstr[d];
  }
}

// Source and destination innermost dimensions differ: each 32 x 32 tile of
// (dimension 0, dimension db) is read along the source's contiguous
// dimension and written along the destination's, through a padded shared
// tile (pitch 33: the column reads of 16-byte values are conflict-free).
__global__ void __launch_bounds__(kTile * kRows) permute_tiled_kernel(PermPlan p, const double2* __restrict__ src,
                                                                     double2* __restrict__ dst) {
  __shared__ double2 t[kTile][kTile + 1];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int64_t na = p.dshape[0], nb = p.dshape[p.db], ldb = p.dstr[p.db], lda = p.sstr[0];
  const int64_t ntile = p.tiles_a * p.tiles_b * p.batch;
  for (int64_t tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
    const int64_t ta = tile % p.tiles_a, rest = tile / p.tiles_a;
    const int64_t tb = rest % p.tiles_b, bi = rest / p.tiles_b;
    int64_t so, dof;
    batch_offsets(p, p.db, bi, so, dof);
    const int64_t a0 = ta * kTile, b0 = tb * kTile;
#pragma unroll
    for (int r = ty; r < kTile; r += kRows) {
      const int64_t a = a0 + r, b = b0 + tx;
      if (a < na && b < nb) t[r][tx] = src[so + a * lda + b];
    }
    __syncthreads();
#pragma unroll
    for (int r = ty; r < kTile; r += kRows) {
      const int64_t a = a0 + tx, b = b0 + r;
      if (a < na && b < nb) dst[dof + a + b * ldb] = t[tx][r];
    }
    __syncthreads();
  }
}

// Source and destination innermost dimensions coincide: contiguous runs of
// dshape[0] elements, one warp row per run chunk.
__global__ void __launch_bounds__(kTile * kRows) permute_rows_kernel(PermPlan p, const double2* __restrict__ src,
                                                                    double2* __restrict__ dst) {
  const int64_t na = p.dshape[0];
  const int64_t chunks = (na + 255) / 256;
  const int64_t total = p.batch * chunks;
  const int t = threadIdx.x + kTile * threadIdx.y;
  for (int64_t w = blockIdx.x; w < total; w += gridDim.x) {
    const int64_t c = w % chunks, bi = w / chunks;
    int64_t so, dof;
    batch_offsets(p, 0, bi, so, dof);
    const int64_t a = c * 256 + t;
    if (a < na) dst[dof + a] = src[so + a];
  }
}

thread_local char g_perm_err[128];

}  // namespace

extern "C" int rgf_permute_c16(rgf_ctx* ctx, const rgf_c16* src, rgf_c16* dst, int32_t ndim,
                               const int64_t* src_shape, const int32_t* order, void* stream) {
  if (!ctx || !src || !dst || !src_shape || !order || ndim < 1 || ndim > kMaxDims) {
    std::snprintf(g_perm_err, sizeof(g_perm_err), "invalid argument");
    return RGF_E_ARG;
  }
  PermPlan p;
  p.nd = ndim;
  int64_t total = 1;
  int64_t src_stride[kMaxDims];
  bool seen[kMaxDims] = {false};
  for (int k = 0; k < ndim; k++) {
    if (src_shape[k] < 1 || order[k] < 1 || order[k] > ndim || seen[order[k] - 1]) {
      std::snprintf(g_perm_err, sizeof(g_perm_err), "shape or order is not a permutation");
      return RGF_E_ARG;
    }
    seen[order[k] - 1] = true;
    src_stride[k] = total;
    total *= src_shape[k];
  }
  for (int k = 0; k < ndim; k++) {
    const int d = order[k] - 1;          // destination dimension fed by source dimension k
    p.dshape[d] = src_shape[k];
    p.sstr[d] = src_stride[k];
  }
  int64_t ds = 1;
  for (int d = 0; d < ndim; d++) {
    p.dstr[d] = ds;
    ds *= p.dshape[d];
  }
  p.db = order[0] - 1;
  int sms = 148, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const dim3 block(kTile, kRows);
  if (p.db == 0) {
    p.tiles_a = p.tiles_b = 1;
    p.batch = total / p.dshape[0];
    const int64_t want = p.batch * ((p.dshape[0] + 255) / 256);
    const unsigned blocks = (unsigned)(want < (int64_t)sms * 16 ? want : (int64_t)sms * 16);
    permute_rows_kernel<<<blocks, block, 0, (cudaStream_t)stream>>>(p, (const double2*)src, (double2*)dst);
  } else {
    p.tiles_a = (p.dshape[0] + kTile - 1) / kTile;
    p.tiles_b = (p.dshape[p.db] + kTile - 1) / kTile;
    p.batch = total / (p.dshape[0] * p.dshape[p.db]);
    const int64_t want = p.tiles_a * p.tiles_b * p.batch;
    const unsigned blocks = (unsigned)(want < (int64_t)sms * 16 ? want : (int64_t)sms * 16);
    permute_tiled_kernel<<<blocks, block, 0, (cudaStream_t)stream>>>(p, (const double2*)src, (double2*)dst);
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    std::snprintf(g_perm_err, sizeof(g_perm_err), "%s", cudaGetErrorString(e));
    return RGF_E_CUDA;
  }
  return RGF_OK;
}

extern "C" const char* rgf_permute_last_error(void) { return g_perm_err; }
