// rgf_gw_fft.cu -- FFT form of the GW loop's energy convolutions, as the
// production loop with energy <-> (i,j) redistribution computes them
// (green_rgf_solve_gw_ephoton_3d_ijs, src/green_rgf.f90:1397-1473 for the
// polarization, :1598-1678 for the self-energy; corr1d2 / conv1d2 with
// method 'fft', src/fft_mod.f90:56-89, :175-212, each a zero-padded
// circular convolution by do_mkl_dfti_conv, :214-234).
//
// The reference forms, for every banded (i,j) element and block ix, one
// length-(2n-1) FFT correlation per (k, q) pair and sums them over k.  Here
// the sums over k move into frequency space: per (i,j, ix) "line" the
// (ky, kz, energy) array of each operand gets one 3-D FFT (energy axis
// zero-padded to N >= 2n-1 with no prime factor above 7), the k - q index
// ikd = k - q + nk/2 - 1 (mod nk) per axis makes the k sums circular
// correlations (P) or convolutions (Sigma) over the k-grid, so
//   P^(p)     = X^(p) Y^(-p) exp(-2 pi i p.s/nk) / (nk N) * dE_P
//   Sigma^(p) = G^(p) W^(p)  exp(+2 pi i p.s/nk) / (nk N) * dE_S
// and one inverse 3-D FFT per output gives every q (or k) at once.  The
// window read back is the 'fft' paths' one: P(p) at energy shift
// b = p - 1 - n/2, Sigma(e) from W placed at nop = -(n/2-1) .. n/2-1.  The
// FFTs are cuFFT's (Z2Z, batched, stream-ordered); packing, the frequency
// products and the window extraction are kernels of this file.
//
// Arrays: the *_by_blocks layout (nen, nk, nx, nij) complex(8) on the device,
// energy fastest, ik = ikz + nkz (iky) (0-based).  nen must be even.
#include <cufft.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <vector>

#include "rgf_internal.h"

namespace {

thread_local char g_fft_err[256];

int fft_fail(int code, const char* msg) {
  std::snprintf(g_fft_err, sizeof(g_fft_err), "%s", msg);
  return code;
}

// smallest m' >= m with no prime factor above 7
int64_t nice_length(int64_t m) {
  for (int64_t n = m;; n++) {
    int64_t r = n;
    for (int64_t p : {2, 3, 5, 7})
      while (r % p == 0) r /= p;
    if (r == 1) return n;
  }
}

struct Dims {
  int64_t nen, nky, nkz, nk, N;
};

// buf[b][k][m] (m < N) from line lines[b] of A: mode 0 the series zero-padded,
// mode 1 its conjugate, mode 2 W placed by energy shift (nop = m for
// m < n/2, nop = m - N for m >= N - (n/2 - 1); W index nop + n/2 - 1).
__global__ void pack_kernel(const double2* __restrict__ A, const int64_t* __restrict__ lines, int64_t nlines,
                            Dims d, int mode, double2* __restrict__ buf) {
  const int64_t total = nlines * d.nk * d.N;
  const int64_t h = d.nen / 2;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t m = t % d.N, r = t / d.N;
    const int64_t k = r % d.nk, b = r / d.nk;
    const double2* src = A + (lines[b] * d.nk + k) * d.nen;
    double2 v = make_double2(0.0, 0.0);
    if (mode == 2) {
      if (m < h) v = src[m + h - 1];
      else if (m >= d.N - (h - 1)) v = src[m - d.N + h - 1];
    } else if (m < d.nen) {
      v = src[m];
      if (mode == 1) v.y = -v.y;
    }
    buf[t] = v;
  }
}

__device__ __forceinline__ double2 cm(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 ca(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }

// P in frequency space, in place over the x-side buffers:
//   xl <- ph (xl ygt~),  xg <- ph (xg ylt~),  xr <- ph (xl ycr~ + xr ylt~)
// with y~ the y-side spectra at negated (ky, kz, energy) frequencies and
// ph[k] the shift phase times the normalisation and dE.
__global__ void corr_freq_kernel(double2* __restrict__ xl, double2* __restrict__ xg, double2* __restrict__ xr,
                                 const double2* __restrict__ ygt, const double2* __restrict__ ylt,
                                 const double2* __restrict__ ycr, const double2* __restrict__ ph, int64_t nlines,
                                 Dims d) {
  const int64_t total = nlines * d.nk * d.N;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t m = t % d.N, r = t / d.N;
    const int64_t k = r % d.nk, b = r / d.nk;
    const int64_t ky = k / d.nkz, kz = k % d.nkz;
    const int64_t kn = ((d.nky - ky) % d.nky) * d.nkz + (d.nkz - kz) % d.nkz;
    const int64_t tn = (b * d.nk + kn) * d.N + (d.N - m) % d.N;
    const double2 p = ph[k];
    const double2 a = xl[t], g = xg[t], rr = xr[t];
    const double2 yl = ylt[tn];
    xl[t] = cm(p, cm(a, ygt[tn]));
    xg[t] = cm(p, cm(g, yl));
    xr[t] = cm(p, ca(cm(a, ycr[tn]), cm(rr, yl)));
  }
}

// Sigma in frequency space, in place over the G-side buffers:
//   gl <- ph gl wl,  gg <- ph gg wg,  gr <- ph (gl wr + gr wl + gr wr)
__global__ void conv_freq_kernel(double2* __restrict__ gl, double2* __restrict__ gg, double2* __restrict__ gr,
                                 const double2* __restrict__ wl, const double2* __restrict__ wg,
                                 const double2* __restrict__ wr, const double2* __restrict__ ph, int64_t nlines,
                                 Dims d) {
  const int64_t total = nlines * d.nk * d.N;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = (t / d.N) % d.nk;
    const double2 p = ph[k];
    const double2 a = gl[t], g = gg[t], rr = gr[t], l = wl[t], w = wr[t];
    gl[t] = cm(p, cm(a, l));
    gg[t] = cm(p, cm(g, wg[t]));
    gr[t] = cm(p, ca(ca(cm(a, w), cm(rr, l)), cm(rr, w)));
  }
}

// outputs of the lines of a chunk: P(o) = buf[(o - n/2) mod N] (mode 0) or
// Sigma(e) = buf[e] with Sigma^R = (Re, Im(Sigma^> - Sigma^<) / 2) (mode 1)
__global__ void unpack_kernel(const double2* __restrict__ b0, const double2* __restrict__ b1,
                              const double2* __restrict__ b2, const int64_t* __restrict__ lines, int64_t nlines,
                              Dims d, int mode, double2* __restrict__ o0, double2* __restrict__ o1,
                              double2* __restrict__ o2) {
  const int64_t total = nlines * d.nk * d.nen;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = t % d.nen, r = t / d.nen;
    const int64_t k = r % d.nk, b = r / d.nk;
    const int64_t src = (b * d.nk + k) * d.N +
                        (mode == 0 ? ((e - d.nen / 2) % d.N + d.N) % d.N : e);
    const int64_t dst = (lines[b] * d.nk + k) * d.nen + e;
    const double2 v0 = b0[src], v1 = b1[src];
    double2 v2 = b2[src];
    if (mode == 1) v2.y = (v1.y - v0.y) / 2.0;
    o0[dst] = v0;
    o1[dst] = v1;
    o2[dst] = v2;
  }
}

struct Plan {
  cufftHandle h = 0;
  bool created = false, ok = false;
  Plan(const Dims& d, int64_t batch, cudaStream_t st) {
    int n[3], rank = 0;
    if (d.nky > 1) n[rank++] = (int)d.nky;
    if (d.nkz > 1) n[rank++] = (int)d.nkz;
    n[rank++] = (int)d.N;
    created = cufftPlanMany(&h, rank, n, nullptr, 1, 0, nullptr, 1, 0, CUFFT_Z2Z, (int)batch) == CUFFT_SUCCESS;
    ok = created && cufftSetStream(h, st) == CUFFT_SUCCESS;
  }
  ~Plan() { if (created) cufftDestroy(h); }
  bool run(double2* buf, int dir) const {
    return cufftExecZ2Z(h, (cufftDoubleComplex*)buf, (cufftDoubleComplex*)buf, dir) == CUFFT_SUCCESS;
  }
};

// Kept in the context between calls (a GW loop calls these every
// iteration): the cuFFT plans of the last shape and the device scratch, so a
// call neither re-plans nor re-allocates.  Freed with the context.
struct FftCache {
  int dev = -1;
  int64_t nky = 0, nkz = 0, N = 0, chunk = 0, tail = 0;
  std::unique_ptr<struct Plan> full, part;
  void* scratch = nullptr;
  size_t bytes = 0;
  ~FftCache();
  static void destroy(void* p) { delete static_cast<FftCache*>(p); }
};

FftCache::~FftCache() {
  full.reset();
  part.reset();
  if (scratch) {
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(dev);
    cudaFree(scratch);
    cudaSetDevice(cur);
  }
}

unsigned grid_for(int64_t total) {
  const int64_t g = (total + 255) / 256;
  return (unsigned)(g < 148 * 32 ? (g < 1 ? 1 : g) : 148 * 32);
}

// mode 0: polarization (x: in[0..2], y: in[3..5]); mode 1: self-energy
// (G: in[0..2], W: in[3..5]).
int run_fft_form(rgf_ctx* ctx, int mode, int64_t nm, int64_t nx, int64_t nen, int64_t nky, int64_t nkz,
                 int64_t ndiag, int64_t nij, int64_t first_ij, double dEn, double spindeg,
                 const double2* const in[6], double2* const out[3], cudaStream_t st) {
  g_fft_err[0] = 0;
  if (nm < 1 || nx < 1 || nen < 2 || (nen % 2) != 0 || nky < 1 || nkz < 1 || ndiag < 0 || nij < 0 ||
      first_ij < 1)
    return fft_fail(RGF_E_ARG, "invalid dimensions (nen must be even and >= 2, first_ij >= 1)");
  for (int a = 0; a < 6; a++)
    if (!in[a]) return fft_fail(RGF_E_ARG, "NULL input array");
  for (int a = 0; a < 3; a++)
    if (!out[a]) return fft_fail(RGF_E_ARG, "NULL output array");
  Dims d;
  d.nen = nen;
  d.nky = nky;
  d.nkz = nkz;
  d.nk = nky * nkz;
  d.N = nice_length(2 * nen - 1);
  if (d.N > (1 << 30) || d.nky > (1 << 20) || d.nkz > (1 << 20))
    return fft_fail(RGF_E_UNSUPPORTED, "transform length out of range");
  const size_t series = (size_t)d.nk * nen;
  // zero every output (elements outside the band stay zero, as the
  // reference's zeroed buffers do)
  for (int a = 0; a < 3; a++) {
    const cudaError_t e = cudaMemsetAsync(out[a], 0, sizeof(double2) * series * nx * nij, st);
    if (e != cudaSuccess) return fft_fail(RGF_E_CUDA, cudaGetErrorString(e));
  }
  // banded lines (i, ix), line = i * nx + ix (src/green_rgf.f90:1401-1408)
  std::vector<int64_t> lines;
  for (int64_t i = 0; i < nij; i++) {
    const int64_t g = i + first_ij;
    const int64_t col = (g - 1) / nm + 1, row = (g - 1) % nm + 1;
    const int64_t lo = row - ndiag > 1 ? row - ndiag : 1, hi = row + ndiag < nm ? row + ndiag : nm;
    if (col < lo || col > hi) continue;
    for (int64_t ix = 0; ix < nx; ix++) lines.push_back(i * nx + ix);
  }
  if (lines.empty()) return RGF_OK;
  // the k-shift phase with the normalisation and dE folded in
  const double kPi = 3.14159265359;   // the reference's pi (src/green_rgf.f90:23)
  double2 dE;
  if (mode == 0) dE = make_double2(0.0, -1.0 * dEn / 2.0 / kPi * spindeg / (double)d.nk);
  else dE = make_double2(0.0, dEn / 2.0 / kPi / (double)d.nk);
  const double norm = 1.0 / ((double)d.nk * (double)d.N);
  const double sgn = mode == 0 ? -1.0 : 1.0;
  const int64_t sy = nky > 1 ? ((nky / 2 - 1) % nky + nky) % nky : 0;
  const int64_t sz = nkz > 1 ? ((nkz / 2 - 1) % nkz + nkz) % nkz : 0;
  std::vector<double2> ph(d.nk);
  for (int64_t k = 0; k < d.nk; k++) {
    const int64_t ky = k / nkz, kz = k % nkz;
    const double th = sgn * 2.0 * M_PI * ((double)(ky * sy) / (double)nky + (double)(kz * sz) / (double)nkz);
    const double2 e = make_double2(std::cos(th) * norm, std::sin(th) * norm);
    ph[k] = make_double2(e.x * dE.x - e.y * dE.y, e.x * dE.y + e.y * dE.x);
  }
  // chunk of lines: six spectra of nk x N complex values each
  const size_t per_line = 6 * (size_t)d.nk * d.N * sizeof(double2);
  int64_t chunk = (int64_t)((size_t)4 << 30) / (int64_t)per_line;
  if (const char* env = std::getenv("RGF_GW_FFT_CHUNK")) {
    const long v = std::atol(env);
    if (v > 0) chunk = v;
  }
  if (chunk < 1) chunk = 1;
  if (chunk > (int64_t)lines.size()) chunk = (int64_t)lines.size();
  const int64_t cap = (int64_t)(0x7fffffff / ((size_t)d.nk * d.N));
  if (chunk > cap) chunk = cap;
  if (chunk < 1) return fft_fail(RGF_E_UNSUPPORTED, "one line exceeds the transform size limit");
  const int64_t nl = (int64_t)lines.size();
  int dev = 0;
  cudaGetDevice(&dev);
  FftCache* cache = static_cast<FftCache*>(rgf::ctx_ext_cache(ctx));
  if (!cache) {
    cache = new FftCache();
    rgf::ctx_set_ext_cache(ctx, cache, &FftCache::destroy);
  }
  const size_t need = per_line * chunk + sizeof(int64_t) * lines.size() + sizeof(double2) * d.nk;
  if (cache->dev != dev || cache->bytes < need) {
    cudaError_t e = cudaStreamSynchronize(st);   // earlier calls may still use the old scratch
    if (cache->scratch) cudaFree(cache->scratch);
    cache->scratch = nullptr;
    cache->bytes = 0;
    if (e == cudaSuccess) e = cudaMalloc(&cache->scratch, need);
    if (e != cudaSuccess) {
      cache->scratch = nullptr;
      return fft_fail(RGF_E_NOMEM, "device scratch for the transforms");
    }
    cache->bytes = need;
  }
  const int64_t tail = nl % chunk;
  if (cache->dev != dev || cache->nky != nky || cache->nkz != nkz || cache->N != d.N || cache->chunk != chunk ||
      cache->tail != tail || !cache->full) {
    cache->full.reset(new Plan(d, chunk, st));
    cache->part.reset(tail ? new Plan(d, tail, st) : nullptr);
    if (!cache->full->ok || (tail && !cache->part->ok)) {
      cache->full.reset();
      cache->part.reset();
      return fft_fail(RGF_E_CUDA, "cuFFT plan");
    }
    cache->dev = dev;
    cache->nky = nky;
    cache->nkz = nkz;
    cache->N = d.N;
    cache->chunk = chunk;
    cache->tail = tail;
  }
  if (cufftSetStream(cache->full->h, st) != CUFFT_SUCCESS ||
      (cache->part && cufftSetStream(cache->part->h, st) != CUFFT_SUCCESS))
    return fft_fail(RGF_E_CUDA, "cuFFT stream");
  const size_t spec = (size_t)chunk * d.nk * d.N;
  double2* buf[6];
  for (int a = 0; a < 6; a++) buf[a] = (double2*)cache->scratch + a * spec;
  int64_t* d_lines = (int64_t*)((double2*)cache->scratch + 6 * spec);
  double2* d_ph = (double2*)(d_lines + lines.size());
  cudaError_t ce = cudaMemcpyAsync(d_lines, lines.data(), sizeof(int64_t) * lines.size(), cudaMemcpyHostToDevice, st);
  if (ce == cudaSuccess) ce = cudaMemcpyAsync(d_ph, ph.data(), sizeof(double2) * d.nk, cudaMemcpyHostToDevice, st);
  if (ce != cudaSuccess) return fft_fail(RGF_E_CUDA, cudaGetErrorString(ce));
  // the host vectors must outlive the asynchronous copies from them
  ce = cudaStreamSynchronize(st);
  if (ce != cudaSuccess) return fft_fail(RGF_E_CUDA, cudaGetErrorString(ce));
  for (int64_t c0 = 0; c0 < nl; c0 += chunk) {
    const int64_t nb = (nl - c0) < chunk ? (nl - c0) : chunk;
    const Plan& plan = nb == chunk ? *cache->full : *cache->part;
    const int64_t* L = d_lines + c0;
    const int64_t tot = nb * d.nk * d.N;
    for (int a = 0; a < 6; a++) {
      const int pm = mode == 0 ? (a == 5 ? 1 : 0) : (a >= 3 ? 2 : 0);
      pack_kernel<<<grid_for(tot), 256, 0, st>>>(in[a], L, nb, d, pm, buf[a]);
      if (!plan.run(buf[a], CUFFT_FORWARD)) return fft_fail(RGF_E_CUDA, "cuFFT forward transform");
    }
    if (mode == 0)
      corr_freq_kernel<<<grid_for(tot), 256, 0, st>>>(buf[0], buf[1], buf[2], buf[3], buf[4], buf[5], d_ph, nb, d);
    else
      conv_freq_kernel<<<grid_for(tot), 256, 0, st>>>(buf[0], buf[1], buf[2], buf[3], buf[4], buf[5], d_ph, nb, d);
    for (int a = 0; a < 3; a++)
      if (!plan.run(buf[a], CUFFT_INVERSE)) return fft_fail(RGF_E_CUDA, "cuFFT inverse transform");
    unpack_kernel<<<grid_for(nb * d.nk * nen), 256, 0, st>>>(buf[0], buf[1], buf[2], L, nb, d, mode, out[0],
                                                             out[1], out[2]);
    ce = cudaGetLastError();
    if (ce != cudaSuccess) return fft_fail(RGF_E_CUDA, cudaGetErrorString(ce));
  }
  ce = cudaStreamSynchronize(st);
  if (ce != cudaSuccess) return fft_fail(RGF_E_CUDA, cudaGetErrorString(ce));
  return RGF_OK;
}

}  // namespace

extern "C" const char* rgf_gw_fft_last_error(void) { return g_fft_err; }

extern "C" int rgf_gw_polarization_fft(rgf_ctx* ctx, int64_t nm, int64_t nx, int64_t nen, int64_t nky,
                                       int64_t nkz, int64_t ndiag, int64_t nij, int64_t first_ij, double dEn,
                                       double spindeg, const rgf_c16* G_lesser, const rgf_c16* G_greater,
                                       const rgf_c16* G_r, const rgf_c16* G_lesser_t,
                                       const rgf_c16* G_greater_t, rgf_c16* P_lesser, rgf_c16* P_greater,
                                       rgf_c16* P_retarded, void* stream) {
  if (!ctx) return fft_fail(RGF_E_ARG, "NULL context");
  // x side: G^<, G^>, G^R; y side: G^>_t, G^<_t, conj(G^R)
  const double2* in[6] = {(const double2*)G_lesser, (const double2*)G_greater, (const double2*)G_r,
                          (const double2*)G_greater_t, (const double2*)G_lesser_t, (const double2*)G_r};
  double2* out[3] = {(double2*)P_lesser, (double2*)P_greater, (double2*)P_retarded};
  return run_fft_form(ctx, 0, nm, nx, nen, nky, nkz, ndiag, nij, first_ij, dEn, spindeg, in, out, (cudaStream_t)stream);
}

extern "C" int rgf_gw_self_energy_fft(rgf_ctx* ctx, int64_t nm, int64_t nx, int64_t nen, int64_t nky,
                                      int64_t nkz, int64_t ndiag, int64_t nij, int64_t first_ij, double dEn,
                                      const rgf_c16* G_lesser, const rgf_c16* G_greater, const rgf_c16* G_r,
                                      const rgf_c16* W_lesser, const rgf_c16* W_greater,
                                      const rgf_c16* W_retarded, rgf_c16* Sigma_lesser_new,
                                      rgf_c16* Sigma_greater_new, rgf_c16* Sigma_r_new, void* stream) {
  if (!ctx) return fft_fail(RGF_E_ARG, "NULL context");
  const double2* in[6] = {(const double2*)G_lesser, (const double2*)G_greater, (const double2*)G_r,
                          (const double2*)W_lesser, (const double2*)W_greater, (const double2*)W_retarded};
  double2* out[3] = {(double2*)Sigma_lesser_new, (double2*)Sigma_greater_new, (double2*)Sigma_r_new};
  return run_fft_form(ctx, 1, nm, nx, nen, nky, nkz, ndiag, nij, first_ij, dEn, 1.0, in, out, (cudaStream_t)stream);
}
