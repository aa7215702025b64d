// rgf_integrals.cu -- energy integrals over the outputs of a batched solve.
//
//   terminal current  sum(tr)*(En(2)-En(1))*e0/tpi/hbar*e0*spindeg/nk
//                     (src/green_rgf.f90:2938, :775, :3189)
//   calc_n_electron   electron / hole density per block from Im G^<_jj and
//                     Im G^>_jj, split at midgap (src/green_rgf.f90:3920-3945)
//
// All are HBM-bound reductions with a fixed thread-to-element mapping and a
// fixed reduction order, so results are bit-reproducible run to run.  They
// run on the legacy default stream (ordered after the caller's work there);
// temporaries are stream-ordered allocations, which neither synchronise the
// device nor return memory to the driver between calls.
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

// calc_n_electron in two passes.  Pass 1: CTA (ix, c) sums chunk c of block
// ix's (energy, k) pairs -- pairs c*per .. (c+1)*per-1 in the order
// i + nen*ik, every diagonal element j of each -- into partial[ix][c]
// (fixed thread mapping and reduction tree).  Pass 2: one thread per block
// adds its chunks in order and applies dE dK.  G arrays (nm,nm,nx,nen,nk)
// column-major.
__global__ void n_electron_partial_kernel(const double2* Gl, const double2* Gg, int64_t nen, const double* E,
                                          int64_t nm, int64_t nk, int64_t nx, int64_t per, const double* midgap,
                                          double2* partial) {
  __shared__ rgf::SmemRed red;
  const int64_t ix = blockIdx.x, c = blockIdx.y, nch = gridDim.y;
  const size_t n2 = (size_t)nm * nm;
  const double mg = midgap[ix];
  const int64_t p0 = c * per, p1 = (p0 + per < nen * nk) ? p0 + per : nen * nk;
  double ne = 0.0, pe = 0.0;
  const int64_t total = (p1 - p0) * nm;
  for (int64_t q = threadIdx.x; q < total; q += rgf::kThreads) {
    const int64_t j = q % nm;
    const int64_t pr = p0 + q / nm;            // pair index i + nen * ik
    const int64_t i = pr % nen, ik = pr / nen;
    const size_t off = (size_t)j * (nm + 1) + ix * n2 + (size_t)nx * n2 * (i + (size_t)nen * ik);
    if (E[i] > mg) ne += Gl[off].y;
    else pe -= Gg[off].y;
  }
  const double2 s = rgf::block_sum2(make_double2(ne, pe), red);
  if (threadIdx.x == 0) partial[ix * nch + c] = s;
}

__global__ void n_electron_combine_kernel(const double2* partial, int64_t nch, int64_t nx, const double* E,
                                          int64_t nk, double* nelec, double* pelec) {
  const int64_t ix = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (ix >= nx) return;
  double ne = 0.0, pe = 0.0;
  for (int64_t c = 0; c < nch; c++) {
    ne += partial[ix * nch + c].x;
    pe += partial[ix * nch + c].y;
  }
  const double dE = (E[1] - E[0]) / (2.0 * kPi);
  const double dK = 2.0 * kPi / (double)nk;
  nelec[ix] = ne * dE * dK;
  pelec[ix] = pe * dE * dK;
}

// calc_block_current (src/green_rgf.f90:4602-4640): one thread per output
// element (io, jo, l); energies summed in the reference's order.  The last
// sub-block of a block repeats the previous one (ib = ns - 1), as the
// reference's stale matrix does; ns = 1 gives zeros.
__global__ void block_current_kernel(const double2* __restrict__ H, const double2* __restrict__ G, int64_t nen,
                                     const double* __restrict__ en, double scale, int64_t nb, int64_t ns,
                                     int64_t nm, int64_t nx, double* __restrict__ tot_cur,
                                     double* __restrict__ tot_ecur, double* __restrict__ jdens) {
  const int64_t b2 = nb * nb, nl = nx * ns;
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= b2 * nl) return;
  const int64_t kk = q % b2, l = q / b2;
  const int64_t io = kk % nb, jo = kk / nb;
  const int64_t ix = l / ns, ibm = l % ns;             // 0-based sub-block index
  const int64_t ib = (ibm == ns - 1) ? ns - 2 : ibm;   // last sub-block repeats the previous one
  const size_t n2 = (size_t)nm * nm;
  double tc = 0.0, te = 0.0;
#pragma unroll 4
  for (int64_t ie = 0; ie < nen; ie++) {
    double v = 0.0;
    if (ib >= 0) {
      const size_t i = io + ib * nb, j = jo + (ib + 1) * nb;
      const double2* Hx = H + ix * n2;
      const double2* Gx = G + ix * n2 + (size_t)ie * nx * n2;
      const double2 b = rgf::csub(rgf::cmul(Hx[i + j * nm], Gx[j + i * nm]), rgf::cmul(Hx[j + i * nm], Gx[i + j * nm]));
      v = b.x * scale;
    }
    if (jdens) jdens[q + (size_t)ie * nl * b2] = v;
    te += en[ie] * v;
    tc += v;
  }
  tot_cur[q] = tc;
  if (tot_ecur) tot_ecur[q] = te;
}

bool is_dev(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Device copy of a (host or device) input array on the legacy default
// stream (stream-ordered allocation); freed, stream-ordered, on destruction.
struct In {
  const void* d = nullptr;
  void* own = nullptr;
  cudaError_t err = cudaSuccess;
  In(const void* p, size_t bytes) {
    if (is_dev(p)) { d = p; return; }
    err = cudaMallocAsync(&own, bytes, 0);
    if (err == cudaSuccess) err = cudaMemcpyAsync(own, p, bytes, cudaMemcpyHostToDevice, 0);
    d = own;
  }
  ~In() { if (own) cudaFreeAsync(own, 0); }
};

// Stream-ordered device scratch of `bytes` (legacy default stream).
struct Tmp {
  void* p = nullptr;
  cudaError_t err;
  explicit Tmp(size_t bytes) { err = cudaMallocAsync(&p, bytes, 0); }
  ~Tmp() { if (p) cudaFreeAsync(p, 0); }
};

}  // namespace

extern "C" int rgf_terminal_current(rgf_ctx* ctx, const double* tr, int64_t nen, double dE,
                                    double spindeg, int64_t nk, double* current) {
  if (!ctx || !tr || !current || nen < 1 || nk < 1) return RGF_E_ARG;
  In x(tr, sizeof(double) * nen);
  if (x.err != cudaSuccess) return RGF_E_CUDA;
  Tmp out(sizeof(double));
  if (out.err != cudaSuccess) return RGF_E_NOMEM;
  sum_kernel<<<1, rgf::kThreads>>>((const double*)x.d, nen, (double*)out.p);
  double s = 0.0;
  const cudaError_t e = cudaMemcpy(&s, out.p, sizeof(double), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return RGF_E_CUDA;
  *current = s * dE * kE0 / kTpi / kHbar * kE0 * spindeg / (double)nk;
  return RGF_OK;
}

extern "C" int rgf_calc_block_current(rgf_ctx* ctx, const rgf_c16* H, const rgf_c16* G_lesser,
                                      int64_t nen, const double* E, double spindeg, int64_t nb,
                                      int64_t ns, int64_t nm, int64_t nx, double* tot_cur,
                                      double* tot_ecur, double* jdens) {
  if (!ctx || !H || !G_lesser || !E || !tot_cur) return RGF_E_ARG;
  if (nen < 2 || nb < 1 || ns < 1 || nm != nb * ns || nx < 1) return RGF_E_ARG;
  const size_t n2 = (size_t)nm * nm;
  In h(H, sizeof(rgf_c16) * n2 * nx), g(G_lesser, sizeof(rgf_c16) * n2 * nx * nen), e(E, sizeof(double) * nen);
  if (h.err || g.err || e.err) return RGF_E_CUDA;
  const size_t nout = (size_t)nb * nb * nx * ns;
  const size_t jbytes = jdens ? sizeof(double) * nout * nen : 0;
  Tmp out(sizeof(double) * 2 * nout + jbytes);
  if (out.err != cudaSuccess) return RGF_E_NOMEM;
  double* d_out = (double*)out.p;
  const double kTpiLocal = 6.28318530718;  // calc_block_current's own tpi (green_rgf.f90:4614)
  const double scale = (E[1] - E[0]) * kE0 / kTpiLocal / kHbar * kE0 * spindeg;
  const int thr = 256;
  const unsigned blocks = (unsigned)((nout + thr - 1) / thr);
  block_current_kernel<<<blocks, thr>>>((const double2*)h.d, (const double2*)g.d, nen, (const double*)e.d,
                                        scale, nb, ns, nm, nx, d_out, d_out + nout,
                                        jdens ? d_out + 2 * nout : nullptr);
  cudaError_t err = cudaMemcpy(tot_cur, d_out, sizeof(double) * nout, cudaMemcpyDeviceToHost);
  if (err == cudaSuccess && tot_ecur) err = cudaMemcpy(tot_ecur, d_out + nout, sizeof(double) * nout, cudaMemcpyDeviceToHost);
  if (err == cudaSuccess && jdens) err = cudaMemcpy(jdens, d_out + 2 * nout, jbytes, cudaMemcpyDeviceToHost);
  return err == cudaSuccess ? RGF_OK : RGF_E_CUDA;
}

extern "C" int rgf_calc_n_electron(rgf_ctx* ctx, const rgf_c16* G_lesser, const rgf_c16* G_greater,
                                   int64_t nen, const double* E, int64_t nm, int64_t nk, int64_t nx,
                                   double* nelec, double* pelec, const double* midgap) {
  if (!ctx || !G_lesser || !G_greater || !E || !nelec || !pelec || !midgap) return RGF_E_ARG;
  if (nen < 2 || nm < 1 || nk < 1 || nx < 1) return RGF_E_ARG;
  const size_t gb = sizeof(rgf_c16) * (size_t)nm * nm * nx * nen * nk;
  In gl(G_lesser, gb), gg(G_greater, gb), e(E, sizeof(double) * nen), mg(midgap, sizeof(double) * nx);
  if (gl.err || gg.err || e.err || mg.err) return RGF_E_CUDA;
  // chunks per block: about four CTAs per SM over the whole grid
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t pairs = nen * nk;
  int64_t nch = (4 * (int64_t)sms + nx - 1) / nx;
  if (nch > pairs) nch = pairs;
  if (nch > 65535) nch = 65535;
  const int64_t per = (pairs + nch - 1) / nch;
  nch = (pairs + per - 1) / per;
  Tmp part(sizeof(double2) * nx * nch), out(2 * sizeof(double) * nx);
  if (part.err != cudaSuccess || out.err != cudaSuccess) return RGF_E_NOMEM;
  n_electron_partial_kernel<<<dim3((unsigned)nx, (unsigned)nch), rgf::kThreads>>>(
      (const double2*)gl.d, (const double2*)gg.d, nen, (const double*)e.d, nm, nk, nx, per,
      (const double*)mg.d, (double2*)part.p);
  double* d_out = (double*)out.p;
  n_electron_combine_kernel<<<(unsigned)((nx + 127) / 128), 128>>>((const double2*)part.p, nch, nx,
                                                                   (const double*)e.d, nk, d_out, d_out + nx);
  cudaError_t err = cudaMemcpy(nelec, d_out, sizeof(double) * nx, cudaMemcpyDeviceToHost);
  if (err == cudaSuccess) err = cudaMemcpy(pelec, d_out + nx, sizeof(double) * nx, cudaMemcpyDeviceToHost);
  return err == cudaSuccess ? RGF_OK : RGF_E_CUDA;
}
