// rgf_integrals.cu -- energy integrals over the outputs of a batched solve.
//
//   terminal current  sum(tr)*(En(2)-En(1))*e0/tpi/hbar*e0*spindeg/nk
//                     (src/green_rgf.f90:2938, :775, :3189)
//   calc_n_electron   electron / hole density per block from Im G^<_jj and
//                     Im G^>_jj, split at midgap (src/green_rgf.f90:3920-3945)
//
// Both are HBM-bound reductions.  Each output value is summed by one CTA with
// a fixed thread-to-element mapping and a fixed reduction tree, so results are
// bit-reproducible run to run.
#include <cstdio>
#include <cstring>
#include <string>

#include "rgf_device.cuh"
#include "rgf_internal.h"

namespace {

constexpr double kE0 = 1.6022e-19;            // green_rgf.f90:22
constexpr double kHbar = 1.0546e-34;          // green_rgf.f90:18
constexpr double kPi = 3.14159265359;         // green_rgf.f90:23
constexpr double kTpi = 3.14159265359 * 2.0;  // green_rgf.f90:24

__global__ void sum_kernel(const double* x, int64_t n, double* out) {
  __shared__ rgf::SmemRed red;
  double acc = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += rgf::kThreads) acc += x[i];
  const double s = rgf::block_sum2(make_double2(acc, 0.0), red).x;
  if (threadIdx.x == 0) *out = s;
}

// One CTA per block ix.  G arrays (nm,nm,nx,nen,nk) column-major.
__global__ void n_electron_kernel(const double2* Gl, const double2* Gg, int64_t nen, const double* E,
                                  int64_t nm, int64_t nk, int64_t nx, const double* midgap,
                                  double* nelec, double* pelec) {
  __shared__ rgf::SmemRed red;
  const int64_t ix = blockIdx.x;
  const size_t n2 = (size_t)nm * nm;
  const double mg = midgap[ix];
  double ne = 0.0, pe = 0.0;
  const int64_t total = nen * nk * nm;
  for (int64_t q = threadIdx.x; q < total; q += rgf::kThreads) {
    const int64_t j = q % nm;
    const int64_t r = q / nm;
    const int64_t ik = r % nk;
    const int64_t i = r / nk;
    const size_t off = (size_t)j * (nm + 1) + ix * n2 + (size_t)nx * n2 * (i + (size_t)nen * ik);
    if (E[i] > mg) ne += Gl[off].y;
    else pe -= Gg[off].y;
  }
  const double2 s = rgf::block_sum2(make_double2(ne, pe), red);
  if (threadIdx.x == 0) {
    const double dE = (E[1] - E[0]) / (2.0 * kPi);
    const double dK = 2.0 * kPi / (double)nk;
    nelec[ix] = s.x * dE * dK;
    pelec[ix] = s.y * dE * dK;
  }
}

bool is_dev(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// device copy of a (host or device) input array; frees on destruction
struct In {
  const void* d = nullptr;
  void* own = nullptr;
  cudaError_t err = cudaSuccess;
  In(const void* p, size_t bytes) {
    if (is_dev(p)) { d = p; return; }
    err = cudaMalloc(&own, bytes);
    if (err == cudaSuccess) err = cudaMemcpy(own, p, bytes, cudaMemcpyHostToDevice);
    d = own;
  }
  ~In() { if (own) cudaFree(own); }
};

}  // namespace

extern "C" int rgf_terminal_current(rgf_ctx* ctx, const double* tr, int64_t nen, double dE,
                                    double spindeg, int64_t nk, double* current) {
  if (!ctx || !tr || !current || nen < 1 || nk < 1) return RGF_E_ARG;
  In x(tr, sizeof(double) * nen);
  if (x.err != cudaSuccess) return RGF_E_CUDA;
  double* d_out = nullptr;
  if (cudaMalloc(&d_out, sizeof(double)) != cudaSuccess) return RGF_E_NOMEM;
  sum_kernel<<<1, rgf::kThreads>>>((const double*)x.d, nen, d_out);
  double s = 0.0;
  cudaError_t e = cudaMemcpy(&s, d_out, sizeof(double), cudaMemcpyDeviceToHost);
  cudaFree(d_out);
  if (e != cudaSuccess) return RGF_E_CUDA;
  *current = s * dE * kE0 / kTpi / kHbar * kE0 * spindeg / (double)nk;
  return RGF_OK;
}

extern "C" int rgf_calc_n_electron(rgf_ctx* ctx, const rgf_c16* G_lesser, const rgf_c16* G_greater,
                                   int64_t nen, const double* E, int64_t nm, int64_t nk, int64_t nx,
                                   double* nelec, double* pelec, const double* midgap) {
  if (!ctx || !G_lesser || !G_greater || !E || !nelec || !pelec || !midgap) return RGF_E_ARG;
  if (nen < 2 || nm < 1 || nk < 1 || nx < 1) return RGF_E_ARG;
  const size_t gb = sizeof(rgf_c16) * (size_t)nm * nm * nx * nen * nk;
  In gl(G_lesser, gb), gg(G_greater, gb), e(E, sizeof(double) * nen), mg(midgap, sizeof(double) * nx);
  if (gl.err || gg.err || e.err || mg.err) return RGF_E_CUDA;
  double* d_out = nullptr;
  if (cudaMalloc(&d_out, 2 * sizeof(double) * nx) != cudaSuccess) return RGF_E_NOMEM;
  n_electron_kernel<<<(unsigned)nx, rgf::kThreads>>>((const double2*)gl.d, (const double2*)gg.d, nen,
                                                     (const double*)e.d, nm, nk, nx,
                                                     (const double*)mg.d, d_out, d_out + nx);
  cudaError_t err = cudaMemcpy(nelec, d_out, sizeof(double) * nx, cudaMemcpyDeviceToHost);
  if (err == cudaSuccess) err = cudaMemcpy(pelec, d_out + nx, sizeof(double) * nx, cudaMemcpyDeviceToHost);
  cudaFree(d_out);
  return err == cudaSuccess ? RGF_OK : RGF_E_CUDA;
}
