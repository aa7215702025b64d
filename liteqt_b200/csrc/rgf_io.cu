// rgf_io.cu -- the reference's spectrum / current / transmission writers
// (src/green_rgf.f90:4541-4896) and the iteration log (:2937-2939), so a
// driver that switches to this library keeps writing identical files.
//
// The sums (diagonal traces per sub-block, current sums) run on the GPU;
// the text is written on the host with an emulation of Fortran's Ew.d and
// Iw edit descriptors: right-justified, mantissa 0.d...d with d digits,
// exponent E+ee (|e| <= 99) or +eee (the E dropped, 99 < |e| <= 999), a '-'
// sign for negative values (negative zero included).  File names are
// dataset // STRING(i) // '.dat' with STRING the reference's 4-digit
// zero-padded number (green.f90:3174-3188), or dataset // '_' // STRING(i)
// for the writers that insert the underscore.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "rgf_device.cuh"
#include "rgf_internal.h"

namespace {

thread_local char g_io_err[256];

int io_fail(int code, const char* msg) {
  std::snprintf(g_io_err, sizeof(g_io_err), "%s", msg);
  return code;
}

bool is_dev(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

struct DevIn {
  const void* d = nullptr;
  void* own = nullptr;
  cudaError_t err = cudaSuccess;
  DevIn(const void* p, size_t bytes) {
    if (is_dev(p)) { d = p; return; }
    err = cudaMalloc(&own, bytes);
    if (err == cudaSuccess) err = cudaMemcpy(own, p, bytes, cudaMemcpyHostToDevice);
    d = own;
  }
  ~DevIn() { if (own) cudaFree(own); }
};

// out[k + NS*(j + length*ie)] = sum_ik sum_ib G(ib+k*NB, ib+k*NB, j, ie, ik); one thread each
__global__ void diag_trace_kernel(const double2* G, int64_t NB, int64_t NS, int64_t length, int64_t nen,
                                  int64_t nk, double2* out) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= NS * length * nen) return;
  const int64_t k = t % NS, j = (t / NS) % length, ie = t / (NS * length);
  const int64_t nm = NB * NS;
  double2 acc = rgf::czero();
  for (int64_t ik = 0; ik < nk; ik++)
    for (int64_t ib = 0; ib < NB; ib++) {
      const int64_t d = ib + k * NB;
      acc = rgf::cadd(acc, G[d + nm * (d + nm * (j + length * (ie + nen * ik)))]);
    }
  out[t] = acc;
}

// out[j + length*ie] = the current sum of one (j, ie) in the loop order of the
// routine: mode 0 ib, jb (write_current_spectrum, :4689-4693); mode 1 ik, ib,
// jb (write_current_spectrum_summed_over_kz, :4725-4733); mode 2 ib, jb, ik
// (write_current_summed_over_k, :4757-4763).  cur(NB, NB, length, nen, nk).
__global__ void cur_sum_kernel(const double* cur, int64_t NB, int64_t length, int64_t nen, int64_t nk,
                               int mode, double* out) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= length * nen) return;
  const int64_t j = t % length, ie = t / length;
  auto at = [&](int64_t ib, int64_t jb, int64_t ik) {
    return cur[ib + NB * (jb + NB * (j + length * (ie + nen * ik)))];
  };
  double acc = 0.0;
  if (mode == 2) {
    for (int64_t ib = 0; ib < NB; ib++)
      for (int64_t jb = 0; jb < NB; jb++)
        for (int64_t ik = 0; ik < nk; ik++) acc += at(ib, jb, ik);
  } else {
    for (int64_t ik = 0; ik < nk; ik++)
      for (int64_t ib = 0; ib < NB; ib++)
        for (int64_t jb = 0; jb < NB; jb++) acc += at(ib, jb, ik);
  }
  out[t] = acc;
}

// DOS of write_dos_summed_over_k (:4832-4840): one running sum per energy
// over j, k, ik, ib in that order
__global__ void dos_kernel(const double2* G, int64_t NB, int64_t NS, int64_t length, int64_t nen, int64_t nk,
                           double2* out) {
  const int64_t ie = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (ie >= nen) return;
  const int64_t nm = NB * NS;
  double2 acc = rgf::czero();
  for (int64_t j = 0; j < length; j++)
    for (int64_t k = 0; k < NS; k++)
      for (int64_t ik = 0; ik < nk; ik++)
        for (int64_t ib = 0; ib < NB; ib++) {
          const int64_t d = ib + k * NB;
          acc = rgf::cadd(acc, G[d + nm * (d + nm * (j + length * (ie + nen * ik)))]);
        }
  out[ie] = acc;
}

// Fortran Ew.d (see the header comment)
std::string fortran_E(double v, int w, int d) {
  char buf[64];
  std::string body;
  if (std::isnan(v) || std::isinf(v)) {
    body = std::isnan(v) ? "NaN" : (v < 0 ? "-Infinity" : "Infinity");
  } else {
    std::snprintf(buf, sizeof(buf), "%.*e", d - 1, std::fabs(v));  // d significant digits
    const char* e = std::strchr(buf, 'e');
    std::string digits;
    for (const char* c = buf; c < e; c++)
      if (*c != '.') digits += *c;
    int ex = std::atoi(e + 1) + 1;
    if (std::fabs(v) == 0.0) ex = 0;
    std::string exps;
    char eb[16];
    if (std::abs(ex) <= 99) {
      std::snprintf(eb, sizeof(eb), "E%c%02d", ex < 0 ? '-' : '+', std::abs(ex));
    } else {
      std::snprintf(eb, sizeof(eb), "%c%03d", ex < 0 ? '-' : '+', std::abs(ex));
    }
    exps = eb;
    body = std::string(std::signbit(v) ? "-" : "") + "0." + digits + exps;
  }
  if ((int)body.size() > w) return std::string(w, '*');
  return std::string(w - body.size(), ' ') + body;
}

std::string fortran_I(long long v, int w) {
  std::string s = std::to_string(v);
  if ((int)s.size() > w) return std::string(w, '*');
  return std::string(w - s.size(), ' ') + s;
}

// STRING(i) (green.f90:3174-3188): 4 digits, zero-padded
std::string fstring(int i) {
  char b[16];
  std::snprintf(b, sizeof(b), "%04d", i);
  return b;
}

FILE* open_out(const std::string& name, int append) { return std::fopen(name.c_str(), append ? "a" : "w"); }

}  // namespace

extern "C" const char* rgf_io_last_error(void) { return g_io_err; }

// write_spectrum (:4541-4573, nk = 1, no division) and
// write_spectrum_summed_over_k (:4771-4810, divided by nk)
extern "C" int rgf_write_spectrum(rgf_ctx* ctx, const char* dataset, int32_t iter, const rgf_c16* G,
                                  int64_t nen, const double* en, int64_t nk, int64_t length, int64_t NB,
                                  int64_t NS, double Lx, const double* coeff, int32_t summed_over_k,
                                  int32_t append) {
  if (!ctx || !dataset || !G || !en || !coeff || nen < 1 || nk < 1 || length < 1 || NB < 1 || NS < 1)
    return io_fail(RGF_E_ARG, "invalid argument");
  const int64_t nm = NB * NS, n = NS * length * nen;
  DevIn g(G, sizeof(rgf_c16) * (size_t)nm * nm * length * nen * nk);
  if (g.err) return io_fail(RGF_E_CUDA, cudaGetErrorString(g.err));
  double2* d_out = nullptr;
  if (cudaMalloc(&d_out, sizeof(double2) * n) != cudaSuccess) return io_fail(RGF_E_NOMEM, "cudaMalloc");
  diag_trace_kernel<<<(unsigned)((n + 255) / 256), 256>>>((const double2*)g.d, NB, NS, length, nen, nk, d_out);
  std::vector<double2> tr(n);
  cudaError_t e = cudaMemcpy(tr.data(), d_out, sizeof(double2) * n, cudaMemcpyDeviceToHost);
  cudaFree(d_out);
  if (e != cudaSuccess) return io_fail(RGF_E_CUDA, cudaGetErrorString(e));
  FILE* f = open_out(std::string(dataset) + fstring(iter) + ".dat", append);
  if (!f) return io_fail(RGF_E_ARG, "cannot open the output file");
  for (int64_t ie = 0; ie < nen; ie++) {
    for (int64_t j = 0; j < length; j++)
      for (int64_t k = 0; k < NS; k++) {
        double2 t = tr[k + NS * (j + length * ie)];
        if (summed_over_k) t = make_double2(t.x / (double)nk, t.y / (double)nk);
        const double x = (double)j * Lx * (double)NS + (double)k * Lx;
        std::fprintf(f, "%s%s%s%s\n", fortran_E(x, 18, 4).c_str(), fortran_E(en[ie], 18, 4).c_str(),
                     fortran_E(t.x * coeff[0], 18, 4).c_str(), fortran_E(t.y * coeff[1], 18, 4).c_str());
      }
    std::fprintf(f, "\n");
  }
  std::fclose(f);
  return RGF_OK;
}

// write_dos_summed_over_k (:4812-4845)
extern "C" int rgf_write_dos(rgf_ctx* ctx, const char* dataset, int32_t iter, const rgf_c16* G, int64_t nen,
                             const double* en, int64_t nk, int64_t length, int64_t NB, int64_t NS, double Lx,
                             int32_t append) {
  if (!ctx || !dataset || !G || !en || nen < 1 || nk < 1 || length < 1 || NB < 1 || NS < 1)
    return io_fail(RGF_E_ARG, "invalid argument");
  const int64_t nm = NB * NS;
  DevIn g(G, sizeof(rgf_c16) * (size_t)nm * nm * length * nen * nk);
  if (g.err) return io_fail(RGF_E_CUDA, cudaGetErrorString(g.err));
  double2* d_out = nullptr;
  if (cudaMalloc(&d_out, sizeof(double2) * nen) != cudaSuccess) return io_fail(RGF_E_NOMEM, "cudaMalloc");
  dos_kernel<<<(unsigned)((nen + 127) / 128), 128>>>((const double2*)g.d, NB, NS, length, nen, nk, d_out);
  std::vector<double2> tr(nen);
  cudaError_t e = cudaMemcpy(tr.data(), d_out, sizeof(double2) * nen, cudaMemcpyDeviceToHost);
  cudaFree(d_out);
  if (e != cudaSuccess) return io_fail(RGF_E_CUDA, cudaGetErrorString(e));
  FILE* f = open_out(std::string(dataset) + fstring(iter) + ".dat", append);
  if (!f) return io_fail(RGF_E_ARG, "cannot open the output file");
  for (int64_t ie = 0; ie < nen; ie++) {
    const double im = tr[ie].y / (double)nk / (double)length / (double)NS / Lx;
    std::fprintf(f, "%s%s\n", fortran_E(en[ie], 18, 4).c_str(), fortran_E(im * (-2.0), 18, 4).c_str());
  }
  std::fclose(f);
  return RGF_OK;
}

// write_current_spectrum (:4681-4702; kz_summed = 0: cur(NB,NB,length,nen),
// dataset_STRING(i), j = 1..length) and write_current_spectrum_summed_over_kz
// (:4707-4745; kz_summed = 1: cur(NB,NB,length,nen,nk), datasetSTRING(i),
// j = 1..length-1, divided by nk)
extern "C" int rgf_write_current_spectrum(rgf_ctx* ctx, const char* dataset, int32_t iter, const double* cur,
                                          int64_t nen, const double* en, int64_t nk, int64_t length,
                                          int64_t NB, double Lx, int32_t kz_summed, int32_t append) {
  if (!ctx || !dataset || !cur || !en || nen < 1 || nk < 1 || length < 1 || NB < 1)
    return io_fail(RGF_E_ARG, "invalid argument");
  const int64_t n = length * nen, nkk = kz_summed ? nk : 1;
  DevIn c(cur, sizeof(double) * (size_t)NB * NB * length * nen * nkk);
  if (c.err) return io_fail(RGF_E_CUDA, cudaGetErrorString(c.err));
  double* d_out = nullptr;
  if (cudaMalloc(&d_out, sizeof(double) * n) != cudaSuccess) return io_fail(RGF_E_NOMEM, "cudaMalloc");
  cur_sum_kernel<<<(unsigned)((n + 255) / 256), 256>>>((const double*)c.d, NB, length, nen, nkk,
                                                       kz_summed ? 1 : 0, d_out);
  std::vector<double> tr(n);
  cudaError_t e = cudaMemcpy(tr.data(), d_out, sizeof(double) * n, cudaMemcpyDeviceToHost);
  cudaFree(d_out);
  if (e != cudaSuccess) return io_fail(RGF_E_CUDA, cudaGetErrorString(e));
  const std::string name = kz_summed ? std::string(dataset) + fstring(iter) + ".dat"
                                     : std::string(dataset) + "_" + fstring(iter) + ".dat";
  FILE* f = open_out(name, kz_summed ? append : 0);
  if (!f) return io_fail(RGF_E_ARG, "cannot open the output file");
  const int64_t jmax = kz_summed ? length - 1 : length;
  for (int64_t ie = 0; ie < nen; ie++) {
    for (int64_t j = 0; j < jmax; j++) {
      double t = tr[j + length * ie];
      if (kz_summed) t = t / (double)nk;
      std::fprintf(f, "%s%s%s\n", fortran_E((double)j * Lx, 18, 4).c_str(), fortran_E(en[ie], 18, 4).c_str(),
                   fortran_E(t, 18, 4).c_str());
    }
    std::fprintf(f, "\n");
  }
  std::fclose(f);
  return RGF_OK;
}

// write_current_summed_over_k (:4748-4768): cur(NB,NB,nx,nk), ii = 1..nx-1
extern "C" int rgf_write_current_summed_over_k(rgf_ctx* ctx, const char* dataset, int32_t iter,
                                               const double* cur, int64_t nx, int64_t NB, double Lx, int64_t nk) {
  if (!ctx || !dataset || !cur || nx < 1 || NB < 1 || nk < 1) return io_fail(RGF_E_ARG, "invalid argument");
  DevIn c(cur, sizeof(double) * (size_t)NB * NB * nx * nk);
  if (c.err) return io_fail(RGF_E_CUDA, cudaGetErrorString(c.err));
  double* d_out = nullptr;
  if (cudaMalloc(&d_out, sizeof(double) * nx) != cudaSuccess) return io_fail(RGF_E_NOMEM, "cudaMalloc");
  // (nb, nb, nx, nk) is the (nb, nb, length = nx, nen = 1, nk) layout
  cur_sum_kernel<<<(unsigned)((nx + 255) / 256), 256>>>((const double*)c.d, NB, nx, 1, nk, 2, d_out);
  std::vector<double> tr(nx);
  cudaError_t e = cudaMemcpy(tr.data(), d_out, sizeof(double) * nx, cudaMemcpyDeviceToHost);
  cudaFree(d_out);
  if (e != cudaSuccess) return io_fail(RGF_E_CUDA, cudaGetErrorString(e));
  FILE* f = open_out(std::string(dataset) + "_" + fstring(iter) + ".dat", 0);
  if (!f) return io_fail(RGF_E_ARG, "cannot open the output file");
  for (int64_t ii = 0; ii < nx - 1; ii++)
    std::fprintf(f, "%s%s\n", fortran_E((double)ii * Lx, 18, 4).c_str(), fortran_E(tr[ii] / (double)nk, 18, 4).c_str());
  std::fclose(f);
  return RGF_OK;
}

// write_transmission_spectrum (:4847-4859; nk = 0: tr(nen), dataset_STRING(i))
// and write_transmission_spectrum_k (:4862-4896; tr(nen,nk) averaged over k,
// datasetSTRING(i)).  Host arrays; O(nen*nk) work.
extern "C" int rgf_write_transmission_spectrum(const char* dataset, int32_t iter, const double* tr, int64_t nen,
                                               const double* en, int64_t nk, int32_t append) {
  if (!dataset || !tr || !en || nen < 1 || nk < 0) return io_fail(RGF_E_ARG, "invalid argument");
  const std::string name = nk > 0 ? std::string(dataset) + fstring(iter) + ".dat"
                                  : std::string(dataset) + "_" + fstring(iter) + ".dat";
  FILE* f = open_out(name, nk > 0 ? append : 0);
  if (!f) return io_fail(RGF_E_ARG, "cannot open the output file");
  for (int64_t ie = 0; ie < nen; ie++) {
    double v = tr[ie];
    if (nk > 0) {
      v = 0.0;
      for (int64_t ik = 0; ik < nk; ik++) v += tr[ie + nen * ik];
      v = v / (double)nk;
    }
    std::fprintf(f, "%s%s\n", fortran_E(en[ie], 18, 4).c_str(), fortran_E(v, 18, 4).c_str());
  }
  std::fclose(f);
  return RGF_OK;
}

// Id_iteration.dat (:2937-2939): '(I4,2E16.6)' iter, I_left, I_right, appended
extern "C" int rgf_write_id_iteration(const char* path, int32_t iter, double current_left, double current_right) {
  if (!path) return io_fail(RGF_E_ARG, "invalid argument");
  FILE* f = std::fopen(path, "a");
  if (!f) return io_fail(RGF_E_ARG, "cannot open the output file");
  std::fprintf(f, "%s%s%s\n", fortran_I(iter, 4).c_str(), fortran_E(current_left, 16, 6).c_str(),
               fortran_E(current_right, 16, 6).c_str());
  std::fclose(f);
  return RGF_OK;
}
