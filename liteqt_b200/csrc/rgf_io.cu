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
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
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

// Device view of a host or device input array.  Copies and temporaries are
// stream-ordered on the legacy default stream (where the sums run, after the
// caller's work there), so a call neither synchronises the device for an
// allocation nor returns memory to the driver.
struct DevIn {
  const void* d = nullptr;
  void* own = nullptr;
  cudaError_t err = cudaSuccess;
  DevIn(const void* p, size_t bytes) {
    if (is_dev(p)) { d = p; return; }
    err = cudaMallocAsync(&own, bytes, 0);
    if (err == cudaSuccess) err = cudaMemcpyAsync(own, p, bytes, cudaMemcpyHostToDevice, 0);
    d = own;
  }
  ~DevIn() { if (own) cudaFreeAsync(own, 0); }
};

struct DevTmp {
  void* p = nullptr;
  cudaError_t err;
  explicit DevTmp(size_t bytes) { err = cudaMallocAsync(&p, bytes, 0); }
  ~DevTmp() { if (p) cudaFreeAsync(p, 0); }
};

// Sum, in index order e = 0 .. count-1, of the values at(e), by one warp:
// the lanes load 32 consecutive terms at a time (the next 32 in flight while
// these are added) and every lane adds them in order, so the result is the
// sequential loop's, bit for bit.
__device__ __forceinline__ double add_lane(double acc, double v, int l) {
  return acc + __shfl_sync(0xffffffffu, v, l);
}
__device__ __forceinline__ double2 add_lane(double2 acc, double2 v, int l) {
  return make_double2(acc.x + __shfl_sync(0xffffffffu, v.x, l), acc.y + __shfl_sync(0xffffffffu, v.y, l));
}
template <class T, class At>
__device__ __forceinline__ T warp_ordered_sum(int64_t count, At at) {
  const int lane = threadIdx.x & 31;
  T acc{};
  T nxt{};
  if (lane < count) nxt = at(lane);
  for (int64_t base = 0; base < count; base += 32) {
    const T cur = nxt;
    if (base + 32 + lane < count) nxt = at(base + 32 + lane);
    const int n = (count - base) < 32 ? (int)(count - base) : 32;
    for (int l = 0; l < n; l++) acc = add_lane(acc, cur, l);
  }
  return acc;
}

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
  const int64_t t = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;   // one warp per output
  if (t >= length * nen) return;
  const int64_t j = t % length, ie = t / length;
  auto at = [&](int64_t ib, int64_t jb, int64_t ik) {
    return cur[ib + NB * (jb + NB * (j + length * (ie + nen * ik)))];
  };
  double acc;
  if (mode == 2) {   // ib, jb, ik (ik fastest)
    acc = warp_ordered_sum<double>(NB * NB * nk, [&](int64_t e) {
      return at(e / (NB * nk), (e / nk) % NB, e % nk);
    });
  } else {           // ik, ib, jb (jb fastest)
    acc = warp_ordered_sum<double>(NB * NB * nk, [&](int64_t e) {
      return at((e / NB) % NB, e % NB, e / (NB * NB));
    });
  }
  if ((threadIdx.x & 31) == 0) out[t] = acc;
}

// DOS of write_dos_summed_over_k (:4832-4840): one running sum per energy
// over j, k, ik, ib in that order (ib fastest); one warp per energy
__global__ void dos_kernel(const double2* G, int64_t NB, int64_t NS, int64_t length, int64_t nen, int64_t nk,
                           double2* out) {
  const int64_t ie = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (ie >= nen) return;
  const int64_t nm = NB * NS;
  const double2 acc = warp_ordered_sum<double2>(length * NS * nk * NB, [&](int64_t e) {
    const int64_t ib = e % NB, r = e / NB;
    const int64_t ik = r % nk, r2 = r / nk;
    const int64_t k = r2 % NS, j = r2 / NS;
    const int64_t d = ib + k * NB;
    return G[d + nm * (d + nm * (j + length * (ie + nen * ik)))];
  });
  if ((threadIdx.x & 31) == 0) out[ie] = acc;
}

// Fortran Ew.d (see the header comment), written as exactly w characters
// into out
void fortran_E_to(char* out, double v, int w, int d) {
  char body[64];
  int n = 0;
  if (std::isnan(v) || std::isinf(v)) {
    const char* t = std::isnan(v) ? "NaN" : (v < 0 ? "-Infinity" : "Infinity");
    n = (int)std::strlen(t);
    std::memcpy(body, t, n);
  } else {
    char buf[64];
    std::snprintf(buf, sizeof(buf), "%.*e", d - 1, std::fabs(v));  // d significant digits
    const char* e = std::strchr(buf, 'e');
    int ex = std::atoi(e + 1) + 1;
    if (std::fabs(v) == 0.0) ex = 0;
    if (std::signbit(v)) body[n++] = '-';
    body[n++] = '0';
    body[n++] = '.';
    for (const char* c = buf; c < e; c++)
      if (*c != '.') body[n++] = *c;
    const int ax = ex < 0 ? -ex : ex;
    if (ax <= 99) {
      body[n++] = 'E';
      body[n++] = ex < 0 ? '-' : '+';
    } else {
      body[n++] = ex < 0 ? '-' : '+';
      body[n++] = (char)('0' + ax / 100);
    }
    body[n++] = (char)('0' + (ax / 10) % 10);
    body[n++] = (char)('0' + ax % 10);
  }
  if (n > w) {
    std::memset(out, '*', w);
    return;
  }
  std::memset(out, ' ', w - n);
  std::memcpy(out + (w - n), body, n);
}

std::string fortran_E(double v, int w, int d) {
  std::string s(w, ' ');
  fortran_E_to(&s[0], v, w, d);
  return s;
}

// append Ew.d to a text buffer
void put_E(std::string& s, double v, int w, int d) {
  const size_t o = s.size();
  s.resize(o + w);
  fortran_E_to(&s[o], v, w, d);
}

bool write_all(FILE* f, const std::string& text) {
  const bool ok = std::fwrite(text.data(), 1, text.size(), f) == text.size();
  return std::fclose(f) == 0 && ok;
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
  DevTmp out(sizeof(double2) * n);
  if (out.err != cudaSuccess) return io_fail(RGF_E_NOMEM, "device scratch");
  double2* d_out = (double2*)out.p;
  diag_trace_kernel<<<(unsigned)((n + 255) / 256), 256>>>((const double2*)g.d, NB, NS, length, nen, nk, d_out);
  std::vector<double2> tr(n);
  cudaError_t e = cudaMemcpy(tr.data(), d_out, sizeof(double2) * n, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return io_fail(RGF_E_CUDA, cudaGetErrorString(e));
  FILE* f = open_out(std::string(dataset) + fstring(iter) + ".dat", append);
  if (!f) return io_fail(RGF_E_ARG, "cannot open the output file");
  std::string text;
  text.reserve((size_t)nen * (length * NS * 73 + 1));
  for (int64_t ie = 0; ie < nen; ie++) {
    for (int64_t j = 0; j < length; j++)
      for (int64_t k = 0; k < NS; k++) {
        double2 t = tr[k + NS * (j + length * ie)];
        if (summed_over_k) t = make_double2(t.x / (double)nk, t.y / (double)nk);
        const double x = (double)j * Lx * (double)NS + (double)k * Lx;
        put_E(text, x, 18, 4);
        put_E(text, en[ie], 18, 4);
        put_E(text, t.x * coeff[0], 18, 4);
        put_E(text, t.y * coeff[1], 18, 4);
        text += '\n';
      }
    text += '\n';
  }
  if (!write_all(f, text)) return io_fail(RGF_E_ARG, "cannot write the output file");
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
  DevTmp out(sizeof(double2) * nen);
  if (out.err != cudaSuccess) return io_fail(RGF_E_NOMEM, "device scratch");
  double2* d_out = (double2*)out.p;
  dos_kernel<<<(unsigned)((32 * nen + 127) / 128), 128>>>((const double2*)g.d, NB, NS, length, nen, nk, d_out);
  std::vector<double2> tr(nen);
  cudaError_t e = cudaMemcpy(tr.data(), d_out, sizeof(double2) * nen, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return io_fail(RGF_E_CUDA, cudaGetErrorString(e));
  FILE* f = open_out(std::string(dataset) + fstring(iter) + ".dat", append);
  if (!f) return io_fail(RGF_E_ARG, "cannot open the output file");
  std::string text;
  for (int64_t ie = 0; ie < nen; ie++) {
    const double im = tr[ie].y / (double)nk / (double)length / (double)NS / Lx;
    put_E(text, en[ie], 18, 4);
    put_E(text, im * (-2.0), 18, 4);
    text += '\n';
  }
  if (!write_all(f, text)) return io_fail(RGF_E_ARG, "cannot write the output file");
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
  DevTmp out(sizeof(double) * n);
  if (out.err != cudaSuccess) return io_fail(RGF_E_NOMEM, "device scratch");
  double* d_out = (double*)out.p;
  cur_sum_kernel<<<(unsigned)((32 * n + 255) / 256), 256>>>((const double*)c.d, NB, length, nen, nkk,
                                                            kz_summed ? 1 : 0, d_out);
  std::vector<double> tr(n);
  cudaError_t e = cudaMemcpy(tr.data(), d_out, sizeof(double) * n, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return io_fail(RGF_E_CUDA, cudaGetErrorString(e));
  const std::string name = kz_summed ? std::string(dataset) + fstring(iter) + ".dat"
                                     : std::string(dataset) + "_" + fstring(iter) + ".dat";
  FILE* f = open_out(name, kz_summed ? append : 0);
  if (!f) return io_fail(RGF_E_ARG, "cannot open the output file");
  const int64_t jmax = kz_summed ? length - 1 : length;
  std::string text;
  for (int64_t ie = 0; ie < nen; ie++) {
    for (int64_t j = 0; j < jmax; j++) {
      double t = tr[j + length * ie];
      if (kz_summed) t = t / (double)nk;
      put_E(text, (double)j * Lx, 18, 4);
      put_E(text, en[ie], 18, 4);
      put_E(text, t, 18, 4);
      text += '\n';
    }
    text += '\n';
  }
  if (!write_all(f, text)) return io_fail(RGF_E_ARG, "cannot write the output file");
  return RGF_OK;
}

// write_current_summed_over_k (:4748-4768): cur(NB,NB,nx,nk), ii = 1..nx-1
extern "C" int rgf_write_current_summed_over_k(rgf_ctx* ctx, const char* dataset, int32_t iter,
                                               const double* cur, int64_t nx, int64_t NB, double Lx, int64_t nk) {
  if (!ctx || !dataset || !cur || nx < 1 || NB < 1 || nk < 1) return io_fail(RGF_E_ARG, "invalid argument");
  DevIn c(cur, sizeof(double) * (size_t)NB * NB * nx * nk);
  if (c.err) return io_fail(RGF_E_CUDA, cudaGetErrorString(c.err));
  DevTmp out(sizeof(double) * nx);
  if (out.err != cudaSuccess) return io_fail(RGF_E_NOMEM, "device scratch");
  double* d_out = (double*)out.p;
  // (nb, nb, nx, nk) is the (nb, nb, length = nx, nen = 1, nk) layout
  cur_sum_kernel<<<(unsigned)((32 * nx + 255) / 256), 256>>>((const double*)c.d, NB, nx, 1, nk, 2, d_out);
  std::vector<double> tr(nx);
  cudaError_t e = cudaMemcpy(tr.data(), d_out, sizeof(double) * nx, cudaMemcpyDeviceToHost);
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

// ------------------------------------------------------------ ham_dat reader
// w90_load_from_file (src/wannierHam.f90:68-130): the Wannier Hamiltonian
// file the drivers read.  Fortran list-directed input: each READ starts at a
// new record and takes as many values as it needs, continuing over records;
// values are separated by blanks or commas.  A `comment` read takes one
// value and skips the rest of its record.
namespace {

struct FortranListReader {
  std::vector<std::string> records;
  size_t rec = 0;
  std::vector<std::string> pending;  // values left in the current record
  bool open(const char* path) {
    FILE* f = std::fopen(path, "r");
    if (!f) return false;
    char buf[4096];
    std::string line;
    while (std::fgets(buf, sizeof(buf), f)) {
      line += buf;
      if (!line.empty() && line.back() == '\n') {
        records.push_back(line);
        line.clear();
      }
    }
    if (!line.empty()) records.push_back(line);
    std::fclose(f);
    return true;
  }
  static std::vector<std::string> split(const std::string& s) {
    std::vector<std::string> v;
    std::string cur;
    for (char c : s) {
      if (c == ' ' || c == '\t' || c == ',' || c == '\n' || c == '\r') {
        if (!cur.empty()) { v.push_back(cur); cur.clear(); }
      } else {
        cur += c;
      }
    }
    if (!cur.empty()) v.push_back(cur);
    return v;
  }
  // one READ statement of n values
  bool read(size_t n, std::vector<std::string>& out) {
    out.clear();
    pending.clear();
    while (out.size() < n) {
      if (pending.empty()) {
        if (rec >= records.size()) return false;
        pending = split(records[rec++]);
        std::reverse(pending.begin(), pending.end());
        continue;
      }
      out.push_back(pending.back());
      pending.pop_back();
    }
    return true;
  }
};

double fortran_real(const std::string& s) {
  std::string t = s;
  for (char& c : t)
    if (c == 'd' || c == 'D') c = 'e';   // Fortran double-precision exponent letter
  return std::strtod(t.c_str(), nullptr);
}

}  // namespace

extern "C" int rgf_read_ham_dat(const char* path, const int32_t* axis, rgf_ham_info* info, rgf_c16* Hr) {
  if (!path || !info) return io_fail(RGF_E_ARG, "invalid argument");
  FortranListReader rd;
  if (!rd.open(path)) return io_fail(RGF_E_ARG, "cannot open the Hamiltonian file");
  std::vector<std::string> v;
  auto bad = [&]() { return io_fail(RGF_E_ARG, "malformed Hamiltonian file"); };
  if (!rd.read(2, v)) return bad();
  std::memset(info, 0, sizeof(*info));
  info->nvb = (int32_t)std::atol(v[0].c_str());
  info->spin_deg = (int32_t)std::atol(v[1].c_str());
  if (!rd.read(1, v)) return bad();  // comment
  double cell[3][3];                 // cell[c] = alpha, beta, gamm
  for (int c = 0; c < 3; c++) {
    if (!rd.read(3, v)) return bad();
    for (int k = 0; k < 3; k++) cell[c][k] = fortran_real(v[k]);
  }
  if (!rd.read(1, v)) return bad();  // comment
  if (axis) {                        // cell(:,:) = cell(:,axis)
    double c2[3][3];
    for (int c = 0; c < 3; c++) {
      if (axis[c] < 1 || axis[c] > 3) return io_fail(RGF_E_ARG, "axis must be a permutation of 1, 2, 3");
      for (int k = 0; k < 3; k++) c2[c][k] = cell[axis[c] - 1][k];
    }
    std::memcpy(cell, c2, sizeof(cell));
  }
  if (!rd.read(1, v)) return bad();
  const long n = std::atol(v[0].c_str());
  if (n < 1) return bad();
  std::vector<double> ham((size_t)n * 7);
  for (long i = 0; i < n; i++) {
    if (!rd.read(7, v)) return bad();
    double row[7];
    for (int k = 0; k < 7; k++) row[k] = fortran_real(v[k]);
    if (axis) {  // ham(:,1:3) = ham(:,axis)
      double r3[3] = {row[axis[0] - 1], row[axis[1] - 1], row[axis[2] - 1]};
      for (int k = 0; k < 3; k++) row[k] = r3[k];
    }
    for (int k = 0; k < 7; k++) ham[(size_t)i * 7 + k] = row[k];
  }
  // integer assignments of reals truncate toward zero, as in the reference
  double mnx = ham[0], mxx = ham[0], mny = ham[1], mxy = ham[1], mxb = ham[3];
  for (long i = 0; i < n; i++) {
    const double* r = &ham[(size_t)i * 7];
    mnx = std::min(mnx, r[0]);
    mxx = std::max(mxx, r[0]);
    mny = std::min(mny, r[1]);
    mxy = std::max(mxy, r[1]);
    mxb = std::max(mxb, r[3]);
  }
  info->xmin = (int32_t)mnx;
  info->xmax = (int32_t)mxx;
  info->ymin = (int32_t)mny;
  info->ymax = (int32_t)mxy;
  info->nb = (int32_t)mxb;
  info->nx = info->xmax - info->xmin + 1;
  info->ny = info->ymax - info->ymin + 1;
  info->n_entries = (int32_t)n;
  for (int c = 0; c < 3; c++)
    for (int k = 0; k < 3; k++) info->cell[k + 3 * c] = cell[c][k];
  auto dot = [](const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
  auto cross = [](const double* a, const double* b, double* o) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
  };
  const double *alpha = cell[0], *beta = cell[1], *gamm = cell[2];
  const double na = std::sqrt(dot(alpha, alpha));
  double xhat[3] = {alpha[0] / na, alpha[1] / na, alpha[2] / na}, yhat[3];
  cross(xhat, gamm, yhat);
  for (double& y : yhat) y = -y;
  const double ny_ = std::sqrt(dot(yhat, yhat));
  for (double& y : yhat) y = y / ny_;
  info->Ly = std::fabs(dot(beta, yhat));
  info->Lx = std::fabs(dot(alpha, xhat));
  info->Lz = std::sqrt(dot(gamm, gamm));
  double t[3];
  cross(beta, gamm, t);
  const double d1 = dot(alpha, t);
  for (int k = 0; k < 3; k++) info->b1[k] = t[k] / d1;
  cross(gamm, alpha, t);
  const double d2 = dot(beta, t);
  for (int k = 0; k < 3; k++) info->b2[k] = t[k] / d2;
  if (Hr) {
    const int64_t nb = info->nb, nx = info->nx, ny = info->ny;
    std::memset(Hr, 0, sizeof(rgf_c16) * (size_t)nb * nb * nx * ny);
    for (long i = 0; i < n; i++) {
      const double* r = &ham[(size_t)i * 7];
      const int64_t a = (int64_t)std::floor(r[3]) - 1, b = (int64_t)std::floor(r[4]) - 1;
      const int64_t x = (int64_t)std::floor(r[0]) - info->xmin, y = (int64_t)std::floor(r[1]) - info->ymin;
      if (a < 0 || a >= nb || b < 0 || b >= nb || x < 0 || x >= nx || y < 0 || y >= ny)
        return io_fail(RGF_E_ARG, "orbital or cell index out of range in the Hamiltonian file");
      rgf_c16& h = Hr[a + nb * (b + nb * (x + nx * y))];
      h.re = r[5];
      h.im = r[6];
    }
  }
  return RGF_OK;
}
