// rgf_permute.cu -- the local transposes of the GW loop's energy <-> (i,j)
// redistribution (energies_to_ijs_2 / ijs_to_energies_2,
// src/green_rgf.f90:243-329): dst = RESHAPE(src, dst_shape, ORDER=order) of a
// complex(8) array, the Fortran intrinsic's meaning (src taken in array
// element order, dst filled with its subscripts running in the order
// order(1), order(2), ...), for pure transposes: dst_shape(order(k)) =
// src_shape(k).  HBM-bound: one thread per destination element (coalesced
// stores), source index from the permuted strides.
#include <cstdint>
#include <cstdio>

#include <cuda_runtime.h>

#include "rgf_internal.h"

namespace {

constexpr int kMaxDims = 8;

struct PermDims {
  int32_t nd;
  int64_t dst_shape[kMaxDims];
  int64_t src_stride_for_dst_dim[kMaxDims];  // source stride of each destination dimension
  int64_t total;
};

__global__ void permute_kernel(PermDims p, const double2* __restrict__ src, double2* __restrict__ dst) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < p.total; t += stride) {
    int64_t r = t, s = 0;
    for (int d = 0; d < p.nd; d++) {
      const int64_t q = r % p.dst_shape[d];
      r /= p.dst_shape[d];
      s += q * p.src_stride_for_dst_dim[d];
    }
    dst[t] = src[s];
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
  PermDims p;
  p.nd = ndim;
  p.total = 1;
  int64_t src_stride[kMaxDims];
  bool seen[kMaxDims] = {false};
  for (int k = 0; k < ndim; k++) {
    if (src_shape[k] < 1 || order[k] < 1 || order[k] > ndim || seen[order[k] - 1]) {
      std::snprintf(g_perm_err, sizeof(g_perm_err), "shape or order is not a permutation");
      return RGF_E_ARG;
    }
    seen[order[k] - 1] = true;
    src_stride[k] = p.total;
    p.total *= src_shape[k];
  }
  for (int k = 0; k < ndim; k++) {
    const int d = order[k] - 1;          // destination dimension fed by source dimension k
    p.dst_shape[d] = src_shape[k];
    p.src_stride_for_dst_dim[d] = src_stride[k];
  }
  const int threads = 256;
  int sms = 148, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t want = (p.total + threads - 1) / threads;
  const unsigned blocks = (unsigned)(want < (int64_t)sms * 16 ? want : (int64_t)sms * 16);
  permute_kernel<<<blocks, threads, 0, (cudaStream_t)stream>>>(p, (const double2*)src, (double2*)dst);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    std::snprintf(g_perm_err, sizeof(g_perm_err), "%s", cudaGetErrorString(e));
    return RGF_E_CUDA;
  }
  return RGF_OK;
}

extern "C" const char* rgf_permute_last_error(void) { return g_perm_err; }
