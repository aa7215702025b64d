// rgf_gw.cu -- the energy/k convolutions of the GW loop of
// green_rgf_solve_gw_3d (src/green_rgf.f90:2944-3092):
//
//   P^<_ij(w)  = dE_P sum_k sum_E G^<_ij(E,k) G^>_ji(E-w,k-q)
//   P^>_ij(w)  = dE_P sum_k sum_E G^>_ij(E,k) G^<_ji(E-w,k-q)
//   P^R_ij(w)  = dE_P sum_k sum_E G^<_ij(E,k) conj(G^R_ij(E-w,k-q)) + G^R_ij(E,k) G^<_ji(E-w,k-q)
//   S^<>_ij(E) = dE_S sum_w sum_q G^<>_ij(E-w,k-q) W^<>_ij(w,q)
//   S^R_ij(E)  = dE_S sum_w sum_q G^<_ij W^R_ij + G^R_ij W^<_ij + G^R_ij W^R_ij
//
// for |i - j| <= ndiag, dE_P = -i dE/(2 pi) spindeg/nk, dE_S = i dE/(2 pi)/nk,
// followed for S by the reference's Sigma^R imaginary part from
// Sigma^> - Sigma^<, symmetrisation, mixing into the running self-energies
// and the edge-block copies.  These are direct sums, as in the reference:
// every output element is accumulated by one thread in the reference's
// order (P: k then E; S: w then q).  Layout (nm,nm,nx,nen,nk) column-major,
// k = kz + ky*nkz.
//
// Memory pattern: when an element's energy series fit in shared memory
// (6 nen complex values for P, 6 nen nk for S, up to 200 KB) a CTA stages
// them once and sums from shared memory (the *_staged kernels); otherwise
// the direct kernels have a warp take 32 consecutive energy offsets w (P) or
// energies E (S) of one element, so one operand is the same address across
// the warp and the other slides along the energy axis.
#include <cstdio>

#include "rgf_device.cuh"
#include "rgf_internal.h"

namespace {

constexpr double kPiGW = 3.14159265359;  // green_rgf.f90:23
constexpr int kGWThreads = 128;

struct GWDims {
  int64_t nm, nx, nen, nky, nkz, ndiag, nopmax;
  __device__ __forceinline__ size_t at(int64_t i, int64_t j, int64_t ix, int64_t ie, int64_t ik) const {
    return (size_t)i + (size_t)nm * ((size_t)j + (size_t)nm * ((size_t)ix + (size_t)nx * ((size_t)ie + (size_t)nen * ik)));
  }
  // 0-based k - q with the reference's nk/2 shift (green_rgf.f90:2968-2977)
  __device__ __forceinline__ int64_t kd(int64_t ik, int64_t iq) const {
    const int64_t iky = ik / nkz, ikz = ik % nkz, iqy = iq / nkz, iqz = iq % nkz;
    int64_t ikzd = ikz - iqz + nkz / 2, ikyd = iky - iqy + nky / 2;   // 0-based: the reference's value - 1
    ikzd -= 1;
    ikyd -= 1;
    if (ikzd < 0) ikzd += nkz;
    if (ikzd >= nkz) ikzd -= nkz;
    if (ikyd < 0) ikyd += nky;
    if (ikyd >= nky) ikyd -= nky;
    if (nky == 1) ikyd = 0;
    if (nkz == 1) ikzd = 0;
    return ikzd + ikyd * nkz;
  }
};

__device__ __forceinline__ double2 gread(const double2* G, size_t k, int imag_only) {
  const double2 v = G[k];
  return imag_only ? make_double2(0.0 * v.x, v.y) : v;
}

__device__ __forceinline__ double2 cfma(double2 acc, double2 a, double2 b) {
  return rgf::cadd(acc, rgf::cmul(a, b));
}

// grid: x = chunks of energy offsets, y = band element (i, jb), z = ix + nx*iq
__global__ void __launch_bounds__(kGWThreads) gw_p_kernel(GWDims d, int imag_only, double2 scale,
                                                           const double2* GL, const double2* GG,
                                                           const double2* GR, double2* PL, double2* PG,
                                                           double2* PR) {
  const int64_t nop = -d.nopmax + (int64_t)blockIdx.x * kGWThreads + threadIdx.x;
  if (nop > d.nopmax) return;
  const int64_t i = blockIdx.y % d.nm, jb = blockIdx.y / d.nm;
  const int64_t j = i - d.ndiag + jb;
  if (j < 0 || j >= d.nm) return;
  const int64_t ix = blockIdx.z % d.nx, iq = blockIdx.z / d.nx;
  const int64_t nk = d.nky * d.nkz;
  const int64_t iop = nop + d.nen / 2 - 1;            // 0-based energy index of w
  double2 al = rgf::czero(), ag = rgf::czero(), ar = rgf::czero();
  const int64_t lo = (nop + 1 > 1 ? nop + 1 : 1) - 1;  // 0-based E range [lo, hi)
  const int64_t hi = d.nen < d.nen + nop ? d.nen : d.nen + nop;
  for (int64_t ik = 0; ik < nk; ik++) {
    const int64_t ikd = d.kd(ik, iq);
    for (int64_t ie = lo; ie < hi; ie++) {
      const size_t a = d.at(i, j, ix, ie, ik);
      const size_t bt = d.at(j, i, ix, ie - nop, ikd);
      const size_t b = d.at(i, j, ix, ie - nop, ikd);
      const double2 gl = gread(GL, a, imag_only), gg = gread(GG, a, imag_only), gr = gread(GR, a, imag_only);
      const double2 glt = gread(GL, bt, imag_only);
      al = cfma(al, gl, gread(GG, bt, imag_only));
      ag = cfma(ag, gg, glt);
      ar = rgf::cadd(ar, rgf::cadd(rgf::cmul(gl, rgf::cconj(gread(GR, b, imag_only))), rgf::cmul(gr, glt)));
    }
  }
  const size_t o = d.at(i, j, ix, iop, iq);
  PL[o] = rgf::cmul(al, scale);
  PG[o] = rgf::cmul(ag, scale);
  PR[o] = rgf::cmul(ar, scale);
}

// grid: x = chunks of energies, y = band element (i, jb), z = ix + nx*ik
__global__ void __launch_bounds__(kGWThreads) gw_s_kernel(GWDims d, int imag_only, double2 scale,
                                                           const double2* GL, const double2* GG,
                                                           const double2* GR, const double2* WL,
                                                           const double2* WG, const double2* WR,
                                                           double2* NL, double2* NG, double2* NR) {
  const int64_t ie1 = (int64_t)blockIdx.x * kGWThreads + threadIdx.x + 1;  // 1-based E index
  if (ie1 > d.nen) return;
  const int64_t i = blockIdx.y % d.nm, jb = blockIdx.y / d.nm;
  const int64_t j = i - d.ndiag + jb;
  if (j < 0 || j >= d.nm) return;
  const int64_t ix = blockIdx.z % d.nx, ik = blockIdx.z / d.nx;
  const int64_t nk = d.nky * d.nkz;
  double2 al = rgf::czero(), ag = rgf::czero(), ar = rgf::czero();
  for (int64_t nop = -d.nopmax; nop <= d.nopmax; nop++) {
    if (!(ie1 > (nop > 1 ? nop : 1) && ie1 < d.nen + nop)) continue;   // green_rgf.f90:3034
    const int64_t iop = nop + d.nen / 2 - 1;
    for (int64_t iq = 0; iq < nk; iq++) {
      const size_t g = d.at(i, j, ix, ie1 - nop - 1, d.kd(ik, iq));
      const size_t w = d.at(i, j, ix, iop, iq);
      const double2 gl = gread(GL, g, imag_only), gr = gread(GR, g, imag_only);
      const double2 wl = WL[w], wr = WR[w];
      al = cfma(al, gl, wl);
      ag = cfma(ag, gread(GG, g, imag_only), WG[w]);
      ar = rgf::cadd(ar, rgf::cadd(rgf::cadd(rgf::cmul(gl, wr), rgf::cmul(gr, wl)), rgf::cmul(gr, wr)));
    }
  }
  const size_t o = d.at(i, j, ix, ie1 - 1, ik);
  NL[o] = rgf::cmul(al, scale);
  NG[o] = rgf::cmul(ag, scale);
  NR[o] = rgf::cmul(ar, scale);
}

// Shared-memory staged forms of the two sums, used when the staged energy
// series fit: a CTA owns one banded element (i, j, ix) and one q (P) or k
// (Sigma) and all its energy offsets / energies (NPT per thread).  The
// operands that the direct kernels read scattered along the energy axis are
// read once per CTA into shared memory; every output keeps the reference's
// order of summation (P: k, then E; Sigma: w, then q).
constexpr int kStThreads = 256;

template <int NPT>
__global__ void __launch_bounds__(kStThreads) gw_p_staged_kernel(GWDims d, int imag_only, double2 scale,
                                                                  const double2* GL, const double2* GG,
                                                                  const double2* GR, double2* PL, double2* PG,
                                                                  double2* PR) {
  extern __shared__ __align__(16) double2 sh[];
  const int64_t nen = d.nen;
  double2 *aL = sh, *aG = sh + nen, *aR = sh + 2 * nen, *bG = sh + 3 * nen, *bL = sh + 4 * nen,
          *bR = sh + 5 * nen;
  const int64_t i = blockIdx.x % d.nm, jb = blockIdx.x / d.nm;
  const int64_t j = i - d.ndiag + jb;
  if (j < 0 || j >= d.nm) return;                      // uniform over the CTA
  const int64_t ix = blockIdx.y, iq = blockIdx.z;
  const int64_t nk = d.nky * d.nkz;
  double2 al[NPT], ag[NPT], ar[NPT];
#pragma unroll
  for (int c = 0; c < NPT; c++) al[c] = ag[c] = ar[c] = rgf::czero();
  for (int64_t ik = 0; ik < nk; ik++) {
    const int64_t ikd = d.kd(ik, iq);
    __syncthreads();
    for (int64_t e = threadIdx.x; e < nen; e += kStThreads) {
      const size_t a = d.at(i, j, ix, e, ik), bt = d.at(j, i, ix, e, ikd), b = d.at(i, j, ix, e, ikd);
      aL[e] = gread(GL, a, imag_only);
      aG[e] = gread(GG, a, imag_only);
      aR[e] = gread(GR, a, imag_only);
      bG[e] = gread(GG, bt, imag_only);
      bL[e] = gread(GL, bt, imag_only);
      bR[e] = gread(GR, b, imag_only);
    }
    __syncthreads();
#pragma unroll
    for (int c = 0; c < NPT; c++) {
      const int64_t nop = -d.nopmax + threadIdx.x + (int64_t)kStThreads * c;
      if (nop > d.nopmax) continue;
      const int64_t lo = (nop + 1 > 1 ? nop + 1 : 1) - 1;
      const int64_t hi = d.nen < d.nen + nop ? d.nen : d.nen + nop;
      for (int64_t ie = lo; ie < hi; ie++) {
        const int64_t e2 = ie - nop;
        const double2 gl = aL[ie], glt = bL[e2];
        al[c] = cfma(al[c], gl, bG[e2]);
        ag[c] = cfma(ag[c], aG[ie], glt);
        ar[c] = rgf::cadd(ar[c], rgf::cadd(rgf::cmul(gl, rgf::cconj(bR[e2])), rgf::cmul(aR[ie], glt)));
      }
    }
  }
#pragma unroll
  for (int c = 0; c < NPT; c++) {
    const int64_t nop = -d.nopmax + threadIdx.x + (int64_t)kStThreads * c;
    if (nop > d.nopmax) continue;
    const size_t o = d.at(i, j, ix, nop + d.nen / 2 - 1, iq);
    PL[o] = rgf::cmul(al[c], scale);
    PG[o] = rgf::cmul(ag[c], scale);
    PR[o] = rgf::cmul(ar[c], scale);
  }
}

template <int NPT>
__global__ void __launch_bounds__(kStThreads) gw_s_staged_kernel(GWDims d, int imag_only, double2 scale,
                                                                  const double2* GL, const double2* GG,
                                                                  const double2* GR, const double2* WL,
                                                                  const double2* WG, const double2* WR,
                                                                  double2* NL, double2* NG, double2* NR) {
  extern __shared__ __align__(16) double2 sh[];
  const int64_t nen = d.nen, nk = d.nky * d.nkz, ne = nen * nk;
  double2 *gL = sh, *gG = sh + ne, *gR = sh + 2 * ne, *wL = sh + 3 * ne, *wG = sh + 4 * ne, *wR = sh + 5 * ne;
  const int64_t i = blockIdx.x % d.nm, jb = blockIdx.x / d.nm;
  const int64_t j = i - d.ndiag + jb;
  if (j < 0 || j >= d.nm) return;
  const int64_t ix = blockIdx.y, ik = blockIdx.z;
  // g(e, q) = G(i,j,ix,e,k-q), w(e, q) = W(i,j,ix,e,q) for every q
  for (int64_t t = threadIdx.x; t < ne; t += kStThreads) {
    const int64_t e = t % nen, iq = t / nen;
    const size_t g = d.at(i, j, ix, e, d.kd(ik, iq)), w = d.at(i, j, ix, e, iq);
    gL[t] = gread(GL, g, imag_only);
    gG[t] = gread(GG, g, imag_only);
    gR[t] = gread(GR, g, imag_only);
    wL[t] = WL[w];
    wG[t] = WG[w];
    wR[t] = WR[w];
  }
  __syncthreads();
  double2 al[NPT], ag[NPT], ar[NPT];
#pragma unroll
  for (int c = 0; c < NPT; c++) al[c] = ag[c] = ar[c] = rgf::czero();
  for (int64_t nop = -d.nopmax; nop <= d.nopmax; nop++) {
    const int64_t iop = nop + nen / 2 - 1;
    for (int64_t iq = 0; iq < nk; iq++) {
      const double2 wl = wL[iop + nen * iq], wg = wG[iop + nen * iq], wr = wR[iop + nen * iq];
#pragma unroll
      for (int c = 0; c < NPT; c++) {
        const int64_t ie1 = 1 + threadIdx.x + (int64_t)kStThreads * c;
        if (ie1 > nen || !(ie1 > (nop > 1 ? nop : 1) && ie1 < nen + nop)) continue;
        const int64_t g = ie1 - nop - 1 + nen * iq;
        const double2 gl = gL[g], gr = gR[g];
        al[c] = cfma(al[c], gl, wl);
        ag[c] = cfma(ag[c], gG[g], wg);
        ar[c] = rgf::cadd(ar[c], rgf::cadd(rgf::cadd(rgf::cmul(gl, wr), rgf::cmul(gr, wl)), rgf::cmul(gr, wr)));
      }
    }
  }
#pragma unroll
  for (int c = 0; c < NPT; c++) {
    const int64_t ie1 = 1 + threadIdx.x + (int64_t)kStThreads * c;
    if (ie1 > nen) continue;
    const size_t o = d.at(i, j, ix, ie1 - 1, ik);
    NL[o] = rgf::cmul(al[c], scale);
    NG[o] = rgf::cmul(ag[c], scale);
    NR[o] = rgf::cmul(ar[c], scale);
  }
}

constexpr size_t kGWStagedSmemMax = 200 * 1024;

// Launch a staged kernel with NPT = the smallest of 1, 2, 4, 8 covering
// `count` values per CTA; false if none fits (the caller then uses the
// direct kernel).
template <class L1, class L2, class L4, class L8>
bool launch_npt(int64_t count, size_t smem, L1 l1, L2 l2, L4 l4, L8 l8) {
  if (smem > kGWStagedSmemMax) return false;
  const int64_t npt = (count + kStThreads - 1) / kStThreads;
  if (npt <= 1) l1(); else if (npt <= 2) l2(); else if (npt <= 4) l4(); else if (npt <= 8) l8(); else return false;
  return true;
}

// Sigma^R imaginary part from Sigma^> - Sigma^<, symmetrisation and mixing
// (green_rgf.f90:3068-3085); one thread per element of the whole arrays.
__global__ void gw_s_post_kernel(int64_t nm, int64_t total, double alpha, const double2* NL,
                                 const double2* NG, const double2* NR, double2* SL, double2* SG,
                                 double2* SR) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= total) return;
  const int64_t n2 = nm * nm, blk = k / n2, r = k % n2, i = r % nm, j = r / nm;
  const int64_t kt = blk * n2 + j + i * nm;
  auto fixr = [&](int64_t q) { return make_double2(NR[q].x, (NG[q].y - NL[q].y) / 2.0); };
  auto sym = [](double2 a, double2 b) { return make_double2((a.x + b.x) / 2.0, (a.y + b.y) / 2.0); };
  const double2 nr = sym(fixr(k), fixr(kt)), nl = sym(NL[k], NL[kt]), ng = sym(NG[k], NG[kt]);
  auto mix = [&](double2* S, double2 nv) {
    const double2 s = S[k];
    S[k] = rgf::cadd(s, rgf::cscale(rgf::csub(nv, s), alpha));
  };
  mix(SR, nr);
  mix(SL, nl);
  mix(SG, ng);
}

// A(:,:,dst,:,:) = A(:,:,src,:,:) for the three arrays (0-based blocks)
__global__ void gw_copy_block_kernel(int64_t nm, int64_t nx, int64_t nsets, int64_t dst, int64_t src,
                                     double2* A, double2* B, double2* C) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t n2 = nm * nm;
  if (k >= n2 * nsets) return;
  const int64_t set = k / n2, r = k % n2;
  const size_t s = (size_t)r + (size_t)n2 * (src + (size_t)nx * set);
  const size_t t = (size_t)r + (size_t)n2 * (dst + (size_t)nx * set);
  A[t] = A[s];
  B[t] = B[s];
  C[t] = C[s];
}

bool on_device(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// A device view of a caller array: the array itself if it is device memory,
// else a staged copy (copied in if `in`, back to the host by `finish` if `out`).
struct View {
  void* host = nullptr;
  void* dev = nullptr;
  size_t bytes = 0;
  bool own = false, out = false;
  cudaError_t open(void* p, size_t n, bool in, bool o, cudaStream_t st) {
    bytes = n;
    out = o;
    if (on_device(p)) { dev = p; return cudaSuccess; }
    host = p;
    own = true;
    cudaError_t e = cudaMalloc(&dev, n);
    if (e == cudaSuccess && in) e = cudaMemcpyAsync(dev, p, n, cudaMemcpyHostToDevice, st);
    return e;
  }
  cudaError_t finish(cudaStream_t st) {
    return (own && out) ? cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, st) : cudaSuccess;
  }
  ~View() { if (own && dev) cudaFree(dev); }
};

thread_local char g_gw_err[256];

int gw_fail(int code, const char* msg) {
  std::snprintf(g_gw_err, sizeof(g_gw_err), "%s", msg);
  return code;
}

int check_dims(int64_t nm, int64_t nx, int64_t nen, int64_t nky, int64_t nkz, int64_t ndiag) {
  if (nm < 1 || nm > 4096 || nx < 3 || nen < 1 || nky < 1 || nkz < 1 || ndiag < 0)
    return gw_fail(RGF_E_ARG, "invalid GW dimensions (nx >= 3 for the edge-block copies)");
  if (nm * (2 * ndiag + 1) > 65535) return gw_fail(RGF_E_UNSUPPORTED, "nm*(2*ndiag+1) > 65535");
  if (nx * nky * nkz > 65535) return gw_fail(RGF_E_UNSUPPORTED, "nx*nk > 65535");
  return RGF_OK;
}

}  // namespace

extern "C" const char* rgf_gw_last_error(void) { return g_gw_err; }

extern "C" int rgf_gw_polarization(rgf_ctx* ctx, int64_t nm, int64_t nx, int64_t nen, int64_t nky,
                                   int64_t nkz, int64_t ndiag, double dE, double spindeg,
                                   int32_t imag_only, const rgf_c16* G_lesser,
                                   const rgf_c16* G_greater, const rgf_c16* G_r, rgf_c16* P_lesser,
                                   rgf_c16* P_greater, rgf_c16* P_retarded, void* stream) {
  g_gw_err[0] = 0;
  if (!ctx || !G_lesser || !G_greater || !G_r || !P_lesser || !P_greater || !P_retarded)
    return gw_fail(RGF_E_ARG, "NULL argument");
  int rc = check_dims(nm, nx, nen, nky, nkz, ndiag);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t nk = nky * nkz;
  const size_t bytes = sizeof(rgf_c16) * (size_t)nm * nm * nx * nen * nk;
  View gl, gg, gr, pl, pg, pr;
  cudaError_t e = gl.open((void*)G_lesser, bytes, true, false, st);
  if (e == cudaSuccess) e = gg.open((void*)G_greater, bytes, true, false, st);
  if (e == cudaSuccess) e = gr.open((void*)G_r, bytes, true, false, st);
  if (e == cudaSuccess) e = pl.open(P_lesser, bytes, false, true, st);
  if (e == cudaSuccess) e = pg.open(P_greater, bytes, false, true, st);
  if (e == cudaSuccess) e = pr.open(P_retarded, bytes, false, true, st);
  if (e != cudaSuccess) return gw_fail(RGF_E_CUDA, cudaGetErrorString(e));
  for (View* v : {&pl, &pg, &pr}) cudaMemsetAsync(v->dev, 0, bytes, st);
  GWDims d{nm, nx, nen, nky, nkz, ndiag, nen / 2 - 10};
  if (d.nopmax >= 0) {
    const double2 scale = make_double2(0.0, -1.0 * dE / 2.0 / kPiGW * spindeg / (double)nk);
    const double2 *a = (const double2*)gl.dev, *b = (const double2*)gg.dev, *c = (const double2*)gr.dev;
    double2 *o1 = (double2*)pl.dev, *o2 = (double2*)pg.dev, *o3 = (double2*)pr.dev;
    const dim3 sgrid((unsigned)(nm * (2 * ndiag + 1)), (unsigned)nx, (unsigned)nk);
    const size_t smem = 6 * sizeof(double2) * (size_t)nen;
    auto go = [&](auto kern) {
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      kern<<<sgrid, kStThreads, smem, st>>>(d, imag_only, scale, a, b, c, o1, o2, o3);
    };
    const bool staged = launch_npt(
        2 * d.nopmax + 1, smem, [&] { go(gw_p_staged_kernel<1>); }, [&] { go(gw_p_staged_kernel<2>); },
        [&] { go(gw_p_staged_kernel<4>); }, [&] { go(gw_p_staged_kernel<8>); });
    if (!staged) {
      dim3 grid((unsigned)((2 * d.nopmax + 1 + kGWThreads - 1) / kGWThreads), (unsigned)(nm * (2 * ndiag + 1)),
                (unsigned)(nx * nk));
      gw_p_kernel<<<grid, kGWThreads, 0, st>>>(d, imag_only, scale, a, b, c, o1, o2, o3);
    }
  }
  e = cudaGetLastError();
  for (View* v : {&pl, &pg, &pr})
    if (e == cudaSuccess) e = v->finish(st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  return e == cudaSuccess ? RGF_OK : gw_fail(RGF_E_CUDA, cudaGetErrorString(e));
}

extern "C" int rgf_gw_self_energy(rgf_ctx* ctx, int64_t nm, int64_t nx, int64_t nen, int64_t nky,
                                  int64_t nkz, int64_t ndiag, double dE, double alpha_mix,
                                  int32_t imag_only, const rgf_c16* G_lesser, const rgf_c16* G_greater,
                                  const rgf_c16* G_r, const rgf_c16* W_lesser, const rgf_c16* W_greater,
                                  const rgf_c16* W_retarded, rgf_c16* Sigma_lesser_gw,
                                  rgf_c16* Sigma_greater_gw, rgf_c16* Sigma_r_gw, void* stream) {
  g_gw_err[0] = 0;
  if (!ctx || !G_lesser || !G_greater || !G_r || !W_lesser || !W_greater || !W_retarded ||
      !Sigma_lesser_gw || !Sigma_greater_gw || !Sigma_r_gw)
    return gw_fail(RGF_E_ARG, "NULL argument");
  int rc = check_dims(nm, nx, nen, nky, nkz, ndiag);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t nk = nky * nkz;
  const size_t nel = (size_t)nm * nm * nx * nen * nk, bytes = sizeof(rgf_c16) * nel;
  View gl, gg, gr, wl, wg, wr, sl, sg, sr;
  cudaError_t e = gl.open((void*)G_lesser, bytes, true, false, st);
  if (e == cudaSuccess) e = gg.open((void*)G_greater, bytes, true, false, st);
  if (e == cudaSuccess) e = gr.open((void*)G_r, bytes, true, false, st);
  if (e == cudaSuccess) e = wl.open((void*)W_lesser, bytes, true, false, st);
  if (e == cudaSuccess) e = wg.open((void*)W_greater, bytes, true, false, st);
  if (e == cudaSuccess) e = wr.open((void*)W_retarded, bytes, true, false, st);
  if (e == cudaSuccess) e = sl.open(Sigma_lesser_gw, bytes, true, true, st);
  if (e == cudaSuccess) e = sg.open(Sigma_greater_gw, bytes, true, true, st);
  if (e == cudaSuccess) e = sr.open(Sigma_r_gw, bytes, true, true, st);
  double2* nbuf = nullptr;
  if (e == cudaSuccess) e = cudaMalloc(&nbuf, 3 * bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return gw_fail(e == cudaErrorMemoryAllocation ? RGF_E_NOMEM : RGF_E_CUDA, cudaGetErrorString(e));
  }
  cudaMemsetAsync(nbuf, 0, 3 * bytes, st);
  double2 *NL = nbuf, *NG = nbuf + nel, *NR = nbuf + 2 * nel;
  GWDims d{nm, nx, nen, nky, nkz, ndiag, nen / 2 - 10};
  if (d.nopmax >= 0) {
    const double2 scale = make_double2(0.0, dE / 2.0 / kPiGW / (double)nk);
    const double2 *a = (const double2*)gl.dev, *b = (const double2*)gg.dev, *c = (const double2*)gr.dev;
    const double2 *w1 = (const double2*)wl.dev, *w2 = (const double2*)wg.dev, *w3 = (const double2*)wr.dev;
    const dim3 sgrid((unsigned)(nm * (2 * ndiag + 1)), (unsigned)nx, (unsigned)nk);
    const size_t smem = 6 * sizeof(double2) * (size_t)nen * (size_t)nk;
    auto go = [&](auto kern) {
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      kern<<<sgrid, kStThreads, smem, st>>>(d, imag_only, scale, a, b, c, w1, w2, w3, NL, NG, NR);
    };
    const bool staged = launch_npt(
        nen, smem, [&] { go(gw_s_staged_kernel<1>); }, [&] { go(gw_s_staged_kernel<2>); },
        [&] { go(gw_s_staged_kernel<4>); }, [&] { go(gw_s_staged_kernel<8>); });
    if (!staged) {
      dim3 grid((unsigned)((nen + kGWThreads - 1) / kGWThreads), (unsigned)(nm * (2 * ndiag + 1)),
                (unsigned)(nx * nk));
      gw_s_kernel<<<grid, kGWThreads, 0, st>>>(d, imag_only, scale, a, b, c, w1, w2, w3, NL, NG, NR);
    }
  }
  const int tpb = 256;
  gw_s_post_kernel<<<(unsigned)((nel + tpb - 1) / tpb), tpb, 0, st>>>(
      nm, (int64_t)nel, alpha_mix, NL, NG, NR, (double2*)sl.dev, (double2*)sg.dev, (double2*)sr.dev);
  // edge blocks (green_rgf.f90:3087-3092): 1, 2 <- 3, then nx, nx-1 <- nx-2
  const int64_t nsets = nen * nk;
  const unsigned cg = (unsigned)((nm * nm * nsets + tpb - 1) / tpb);
  const int64_t copies[4][2] = {{0, 2}, {1, 2}, {nx - 1, nx - 3}, {nx - 2, nx - 3}};
  for (const auto& c : copies)
    gw_copy_block_kernel<<<cg, tpb, 0, st>>>(nm, nx, nsets, c[0], c[1], (double2*)sr.dev,
                                             (double2*)sl.dev, (double2*)sg.dev);
  e = cudaGetLastError();
  for (View* v : {&sl, &sg, &sr})
    if (e == cudaSuccess) e = v->finish(st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(nbuf);
  return e == cudaSuccess ? RGF_OK : gw_fail(RGF_E_CUDA, cudaGetErrorString(e));
}
