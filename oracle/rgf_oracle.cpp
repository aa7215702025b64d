// rgf_oracle.cpp -- CPU restatement of the reference RGF hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA library in
// liteqt_b200/csrc: it is called by tests/, by __graft_entry__.smoke() and by
// the cpu_baseline / --impl reference legs of bench.py, and by nothing else.
// The product path never links, loads or calls it.
//
// Parity status: the reference (Fortran 90 + MKL) cannot be compiled in this
// environment (no Fortran compiler, no MKL) and ships no tests or golden
// outputs, so this restatement is NOT pinned to outputs of the reference
// itself ("parity unpinned" by reference outputs).  It is pinned instead by
// known answers (dense (E-H-Sigma)^-1 inverse, the Sancho fixed point, the
// integer transmission of a uniform chain, tr = tre current conservation) and
// by an independent NumPy restatement in oracle/oracle.py.
//
// What follows the reference line by line (paths relative to the liteQT tree):
//   green_RGF_RS     src/green_rgf.f90:3950-4164   (rgf_energy below)
//   RGF_G            src/rgf_mod.f90:26-237        (same math, other BOLTZ)
//   sancho           src/green_rgf.f90:4451-4537   (sancho below)
//   invert           src/green_rgf.f90:4421-4441   (invert below)
//   ferm             src/green_rgf.f90:4444-4447   (ferm below)
//   Caroli T(E)      src/green.f90:2571-2580       (transmission, new on the RGF path)
//   calc_n_electron  src/green_rgf.f90:3920-3945
//   terminal current src/green_rgf.f90:2938
//
// Dense arithmetic goes through OpenBLAS (zgemm / zgetrf / zgetri, the build
// bundled with scipy, LP64) opened with dlopen; the library path is handed in
// by the Python wrapper.  These are the same LAPACK algorithms MKL runs
// (partial-pivot LU, getri), so results differ from MKL in the last bits only.

#include <atomic>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <dlfcn.h>
#include <type_traits>
#include <thread>
#include <vector>

typedef std::complex<double> cd;

extern "C" {
typedef void (*zgemm_fn)(const char*, const char*, const int*, const int*, const int*,
                         const cd*, const cd*, const int*, const cd*, const int*,
                         const cd*, cd*, const int*);
typedef void (*zgetrf_fn)(const int*, const int*, cd*, const int*, int*, int*);
typedef void (*zgetri_fn)(const int*, cd*, const int*, const int*, cd*, const int*, int*);
typedef void (*setnt_fn)(int);
}

static zgemm_fn p_zgemm = nullptr;
static zgetrf_fn p_zgetrf = nullptr;
static zgetri_fn p_zgetri = nullptr;
static setnt_fn p_setnt = nullptr;

// Options that select between the reference's exact behaviour ("compat") and
// the physically consistent variants.  Must match struct oracle_opts in oracle.py.
struct OracleOpts {
  double eta_dev;      // device broadening; reference: z = dcmplx(E, 0.0d-6) -> 0  (green_rgf.f90:3974)
  double eta_lead;     // Sancho broadening; reference: 1e-3                       (green_rgf.f90:4474)
  double boltz;        // 8.61734e-5 (green_rgf.f90:3968) or 8.617333262e-5 (parameters.f90:38)
  double sancho_tol;   // 1e-100 (green_rgf.f90:4457)
  int32_t sancho_nmax; // 100 (green_rgf.f90:4473)
  int32_t consistent;  // 0: reference H1i indexing in the backward sweep; 1: H1i(l+1)
  int32_t want_T;      // compute Caroli T(E) with a running G_{N1} product
  int32_t pad;
};

// Counters and status per energy point.  Must match oracle.py.
struct OracleStat {
  int32_t sancho_iters_left;
  int32_t sancho_iters_right;
  int32_t status;       // bit0 singular block, bit1 Sancho not converged
  int32_t n_gemm;       // zgemm calls made
  int32_t n_inv;        // invert calls made
  int32_t pad;
};

enum { ST_SINGULAR = 1, ST_SANCHO_NC = 2, ST_BAD_ARGS = 4 };

extern "C" int oracle_init(const char* blas_path) {
  void* h = dlopen(blas_path, RTLD_NOW | RTLD_LOCAL);
  if (!h) return -1;
  p_zgemm = (zgemm_fn)dlsym(h, "scipy_zgemm_");
  p_zgetrf = (zgetrf_fn)dlsym(h, "scipy_zgetrf_");
  p_zgetri = (zgetri_fn)dlsym(h, "scipy_zgetri_");
  p_setnt = (setnt_fn)dlsym(h, "scipy_openblas_set_num_threads");
  if (!p_zgemm || !p_zgetrf || !p_zgetri) return -2;
  if (p_setnt) p_setnt(1);  // one BLAS thread per call, like libmkl_sequential (Makefile.intel:7)
  return 0;
}

namespace {

// Dense kernels on one scalar type.  double: OpenBLAS zgemm / zgetrf / zgetri
// (the reference's MKL calls).  long double (x87, 64-bit mantissa): plain
// loops and Gauss-Jordan with partial pivoting -- the extended-precision
// ground truth the FP64 results are measured against.
template <typename R>
struct Work {
  typedef std::complex<R> C;
  int nm;
  OracleStat* st;
  std::vector<cd> lu_work;
  std::vector<int> ipiv;
  explicit Work(int n, OracleStat* s) : nm(n), st(s), lu_work((size_t)n * n), ipiv(n) {}

  static C opel(const C* X, char t, int n, int i, int j) {  // op(X)[i][j]
    if (t == 'n') return X[i + (size_t)j * n];
    if (t == 'c') return std::conj(X[j + (size_t)i * n]);
    return X[j + (size_t)i * n];  // 't'
  }

  // C = op(A) * op(B), alpha = 1, beta = 0 (every zgemm of green_RGF_RS)
  void gemm(char ta, char tb, const C* A, const C* B, C* Cm) {
    st->n_gemm++;
    if constexpr (std::is_same<R, double>::value) {
      const cd one(1.0, 0.0), zero(0.0, 0.0);
      p_zgemm(&ta, &tb, &nm, &nm, &nm, &one, A, &nm, B, &nm, &zero, Cm, &nm);
    } else {
      const int n = nm;
      std::vector<C> At((size_t)n * n), Bt((size_t)n * n);
      for (int i = 0; i < n; i++)
        for (int k = 0; k < n; k++) At[k + (size_t)i * n] = opel(A, ta, n, i, k);  // row i contiguous
      for (int j = 0; j < n; j++)
        for (int k = 0; k < n; k++) Bt[k + (size_t)j * n] = opel(B, tb, n, k, j);  // col j contiguous
      for (int j = 0; j < n; j++)
        for (int i = 0; i < n; i++) {
          C acc(0, 0);
          const C* a = &At[(size_t)i * n];
          const C* b = &Bt[(size_t)j * n];
          for (int k = 0; k < n; k++) acc += a[k] * b[k];
          Cm[i + (size_t)j * n] = acc;
        }
    }
  }

  // invert: green_rgf.f90:4421-4441.  zgetrf + zgetri; on info /= 0 the
  // reference prints a warning and returns the zero matrix.
  void invert(C* A) {
    st->n_inv++;
    const int n = nm;
    if constexpr (std::is_same<R, double>::value) {
      int info = 0;
      const int lw = n * n;
      p_zgetrf(&nm, &nm, A, &nm, ipiv.data(), &info);
      if (info == 0) p_zgetri(&nm, A, &nm, ipiv.data(), lu_work.data(), &lw, &info);
      if (info != 0) {
        std::fill(A, A + (size_t)n * n, C(0, 0));
        st->status |= ST_SINGULAR;
      }
    } else {
      std::vector<int> perm(n);
      for (int k = 0; k < n; k++) {
        int p = k;
        R best = -1;
        for (int i = k; i < n; i++) {
          const R v = std::fabs(A[i + (size_t)k * n].real()) + std::fabs(A[i + (size_t)k * n].imag());
          if (v > best) { best = v; p = i; }
        }
        perm[k] = p;
        if (best == 0) {
          std::fill(A, A + (size_t)n * n, C(0, 0));
          st->status |= ST_SINGULAR;
          return;
        }
        if (p != k)
          for (int j = 0; j < n; j++) std::swap(A[k + (size_t)j * n], A[p + (size_t)j * n]);
        const C pinv = C(1, 0) / A[k + (size_t)k * n];
        A[k + (size_t)k * n] = C(1, 0);
        for (int j = 0; j < n; j++) A[k + (size_t)j * n] *= pinv;
        for (int i = 0; i < n; i++) {
          if (i == k) continue;
          const C f = A[i + (size_t)k * n];
          A[i + (size_t)k * n] = C(0, 0);
          for (int j = 0; j < n; j++) A[i + (size_t)j * n] -= f * A[k + (size_t)j * n];
        }
      }
      for (int k = n - 1; k >= 0; k--)
        if (perm[k] != k)
          for (int i = 0; i < n; i++) std::swap(A[i + (size_t)k * n], A[i + (size_t)perm[k] * n]);
    }
  }
};

template <typename R>
inline R ferm(R a) { return R(1) / (R(1) + std::exp(a)); }  // green_rgf.f90:4444-4447

inline size_t nn(int nm) { return (size_t)nm * nm; }

// sancho: green_rgf.f90:4451-4537.  S00 = nullptr is the identity (the
// green_RGF_RS call sites); green_RGF_CMS passes Sii(:,:,1) / Sii(:,:,nx).
// Returns the iteration count taken (nmax+1 encodes "not converged").
template <typename R>
int sancho(Work<R>& w, const OracleOpts& o, R E, const std::complex<R>* S00, const std::complex<R>* H00,
           const std::complex<R>* H10, std::complex<R>* G00, std::complex<R>* GBB) {
  typedef std::complex<R> cd;
  const int nm = w.nm;
  const size_t n2 = nn(nm);
  std::vector<cd> A(n2), B(n2), C(n2), H_BB(H00, H00 + n2), H_SS(H00, H00 + n2),
      H_10(H10, H10 + n2), H_01(n2);
  const cd z(E, (R)o.eta_lead);
  for (int j = 0; j < nm; j++)
    for (int i = 0; i < nm; i++) H_01[i + (size_t)j * nm] = std::conj(H_10[j + (size_t)i * nm]);
  int taken = 0;
  auto zS_minus = [&](const std::vector<cd>& H, cd* out) {  // out = z*S00 - H
    for (size_t k = 0; k < n2; k++) out[k] = (S00 ? z * S00[k] : cd(0, 0)) - H[k];
    if (!S00)
      for (int i = 0; i < nm; i++) out[i + (size_t)i * nm] += z;
  };
  for (int it = 1; it <= o.sancho_nmax; it++) {
    taken = it;
    zS_minus(H_BB, A.data());
    w.invert(A.data());
    w.gemm('n', 'n', A.data(), H_10.data(), B.data());
    w.gemm('n', 'n', H_01.data(), B.data(), C.data());
    for (size_t k = 0; k < n2; k++) { H_SS[k] += C[k]; H_BB[k] += C[k]; }
    w.gemm('n', 'n', H_10.data(), B.data(), C.data());
    w.gemm('n', 'n', A.data(), H_01.data(), B.data());
    w.gemm('n', 'n', H_10.data(), B.data(), A.data());
    H_10 = C;
    for (size_t k = 0; k < n2; k++) H_BB[k] += A[k];
    w.gemm('n', 'n', H_01.data(), B.data(), C.data());
    H_01 = C;
    R error = 0;
    for (size_t k = 0; k < n2; k++)
      error += std::sqrt(C[k].imag() * C[k].imag() + C[k].real() * C[k].real());
    if (std::fabs(error) < o.sancho_tol) break;
    if (it == o.sancho_nmax) {
      H_SS.assign(H00, H00 + n2);
      H_BB.assign(H00, H00 + n2);
      w.st->status |= ST_SANCHO_NC;
      taken = o.sancho_nmax + 1;
    }
  }
  zS_minus(H_SS, G00);
  w.invert(G00);
  zS_minus(H_BB, GBB);
  w.invert(GBB);
  return taken;
}

}  // namespace

// One energy point of green_RGF_RS (green_rgf.f90:3950-4164).
// Arrays are column-major (nm,nm,nx) complex128.  sig_lesser / sig_r may be
// null (treated as zero).  Every output may be null (not written).
// T_out (if non-null, and o.want_T) receives the Caroli transmission
// Re Tr[Gamma_L G^A_{1N} Gamma_R G^R_{N1}] (green.f90:2571-2580).
namespace {

template <typename R>
int rgf_energy(const OracleOpts* opts, int64_t nm64, int64_t nx64, double E_in, const double* mu,
               const double* temp, const cd* Sii_in, const cd* Hii_in, const cd* H1i_in,
               const cd* sig_lesser_in, const cd* sig_r_in, cd* ndens_out, cd* pdens_out,
               cd* ldos_out, double* tr,
               double* tre, double* cur_out, cd* GRi1_out, cd* GLi1_out, cd* GGi1_out,
               double* T_out, OracleStat* st) {
  typedef std::complex<R> cd;
  typedef std::complex<double> cdd;
  const OracleOpts& o = *opts;
  const R E = (R)E_in;
  OracleStat dummy{};
  if (!st) st = &dummy;
  std::memset(st, 0, sizeof(*st));
  if (nm64 < 1 || nx64 < 2 || nm64 > 4096) { st->status = ST_BAD_ARGS; return ST_BAD_ARGS; }
  const int nm = (int)nm64, nx = (int)nx64;
  const size_t n2 = nn(nm);
  Work<R> w(nm, st);
  // inputs and outputs in the working precision
  const size_t nall = n2 * (size_t)nx;
  std::vector<cd> Hii_v(Hii_in, Hii_in + nall), H1i_v(H1i_in, H1i_in + nall), Sii_v;
  if (Sii_in) Sii_v.assign(Sii_in, Sii_in + nall);
  // green_RGF_CMS (green_rgf.f90:4167-4383) when an overlap is given
  const bool cms = Sii_in != nullptr;
  const cd* Sii = cms ? Sii_v.data() : nullptr;
  std::vector<cd> sl_v, sr_v, nd_v, pd_v, ld_v, gr_v, gl_v, gg_v;
  std::vector<R> cur_v;
  if (sig_lesser_in) sl_v.assign(sig_lesser_in, sig_lesser_in + nall);
  if (sig_r_in) sr_v.assign(sig_r_in, sig_r_in + nall);
  auto outbuf = [&](cdd* p, std::vector<cd>& v) -> cd* {
    if (!p) return nullptr;
    v.assign(p, p + nall);  // keep the caller's values where nothing is written
    return v.data();
  };
  const cd* Hii = Hii_v.data();
  const cd* H1i = H1i_v.data();
  const cd* sig_lesser = sig_lesser_in ? sl_v.data() : nullptr;
  const cd* sig_r = sig_r_in ? sr_v.data() : nullptr;
  cd* ndens = outbuf(ndens_out, nd_v);
  cd* pdens = outbuf(pdens_out, pd_v);
  cd* ldos = outbuf(ldos_out, ld_v);
  cd* GRi1 = outbuf(GRi1_out, gr_v);
  cd* GLi1 = outbuf(GLi1_out, gl_v);
  cd* GGi1 = outbuf(GGi1_out, gg_v);
  R* cur = nullptr;
  if (cur_out) { cur_v.assign(cur_out, cur_out + nall); cur = cur_v.data(); }
  auto blk = [&](const cd* base, int l) { return base + (size_t)(l - 1) * n2; };  // 1-based l
  auto blkw = [&](cd* base, int l) { return base + (size_t)(l - 1) * n2; };
  auto adj = [&](const cd* X, cd* Y) {  // Y = X^H
    for (int j = 0; j < nm; j++)
      for (int i = 0; i < nm; i++) Y[i + (size_t)j * nm] = std::conj(X[j + (size_t)i * nm]);
  };
  auto sigR = [&](int l, size_t k) { return sig_r ? blk(sig_r, l)[k] : cd(0.0, 0.0); };
  auto sigL = [&](int l, size_t k) { return sig_lesser ? blk(sig_lesser, l)[k] : cd(0.0, 0.0); };
  // CMS multiplies the scattering self-energies by the overlap block:
  // sigma_r_ph(l) S00 (:4204, :4226) and sigma_lesser_ph(l) S00 (:4211, :4240);
  // RS adds them as they are.  SR[l-1] / SL[l-1] hold the per-block terms.
  std::vector<std::vector<cd>> SRt, SLt;
  if (cms) {
    SRt.assign(nx, std::vector<cd>(n2, cd(0, 0)));
    SLt.assign(nx, std::vector<cd>(n2, cd(0, 0)));
    for (int l = 1; l <= nx; l++) {
      if (sig_r) w.gemm('n', 'n', blk(sig_r, l), blk(Sii, l), SRt[l - 1].data());
      if (sig_lesser) w.gemm('n', 'n', blk(sig_lesser, l), blk(Sii, l), SLt[l - 1].data());
    }
  }
  auto sR = [&](int l, size_t k) { return cms ? SRt[l - 1][k] : sigR(l, k); };
  auto sL = [&](int l, size_t k) { return cms ? SLt[l - 1][k] : sigL(l, k); };
  // The backward sweep's coupling block: reference uses H1i(:,:,l) (trap T3);
  // the consistent variant uses H_{l+1,l} = H1i(:,:,l+1).
  auto H1b = [&](int l) { return o.consistent ? blk(H1i, l + 1) : blk(H1i, l); };

  const R mul = mu[0], mur = mu[1], templ = temp[0], tempr = temp[1];
  const cd z(E, (R)o.eta_dev);
  // A = z*S_ll - X (RS: S = I)
  auto zS = [&](int l, const cd* X, cd* Aout) {
    for (size_t k = 0; k < n2; k++) Aout[k] = (cms ? z * blk(Sii, l)[k] : cd(0, 0)) - X[k];
    if (!cms)
      for (int i = 0; i < nm; i++) Aout[i + (size_t)i * nm] += z;
  };
  std::vector<cd> Gl(n2 * nx), Gln(n2 * nx);
  std::vector<cd> H00(n2), H10(n2), A(n2), B(n2), C(n2), D(n2), G00(n2), GBB(n2), GN0(n2),
      Gn(n2), Gp(n2), sig(n2), sigmal(n2), sigmar(n2), tmp(n2), GN1(n2), GN1b(n2);

  if (ldos) std::fill(ldos, ldos + n2 * nx, cd(0, 0));
  if (ndens) std::fill(ndens, ndens + n2 * nx, cd(0, 0));
  if (pdens) std::fill(pdens, pdens + n2 * nx, cd(0, 0));
  if (cur) std::fill(cur, cur + n2 * nx, R(0));

  // ---- left contact (green_rgf.f90:3992-4012)
  for (size_t k = 0; k < n2; k++) H00[k] = blk(Hii, 1)[k] + sR(1, k);
  std::copy(blk(H1i, 1), blk(H1i, 1) + n2, H10.begin());
  adj(H10.data(), tmp.data());
  st->sancho_iters_left = sancho(w, o, E, cms ? blk(Sii, 1) : nullptr, H00.data(), tmp.data(),
                                 G00.data(), GBB.data());
  w.gemm('n', 'n', H10.data(), G00.data(), A.data());
  w.gemm('n', 'c', A.data(), H10.data(), sigmal.data());
  {
    const R f = ferm<R>((E - mul) / ((R)o.boltz * templ));
    for (int j = 0; j < nm; j++)
      for (int i = 0; i < nm; i++) {
        const size_t k = i + (size_t)j * nm;
        sig[k] = -(sigmal[k] - std::conj(sigmal[j + (size_t)i * nm])) * f + sL(1, k);
      }
  }
  for (size_t k = 0; k < n2; k++) C[k] = H00[k] + sigmal[k];
  zS(1, C.data(), A.data());
  w.invert(A.data());
  std::copy(A.begin(), A.end(), blkw(Gl.data(), 1));
  w.gemm('n', 'n', A.data(), sig.data(), B.data());
  w.gemm('n', 'c', B.data(), A.data(), C.data());
  std::copy(C.begin(), C.end(), blkw(Gln.data(), 1));
  // running left-connected column g^L_{l,1}; g^L_{1,1} = g_1  (for T(E))
  if (o.want_T) GN1 = A;

  // ---- forward sweep (green_rgf.f90:4013-4030)
  for (int l = 2; l <= nx - 1; l++) {
    for (size_t k = 0; k < n2; k++) H00[k] = blk(Hii, l)[k] + sR(l, k);
    std::copy(blk(H1i, l), blk(H1i, l) + n2, H10.begin());
    w.gemm('n', 'n', H10.data(), blkw(Gl.data(), l - 1), B.data());
    w.gemm('n', 'c', B.data(), H10.data(), C.data());
    for (size_t k = 0; k < n2; k++) C[k] += H00[k];
    zS(l, C.data(), A.data());
    w.invert(A.data());
    std::copy(A.begin(), A.end(), blkw(Gl.data(), l));
    std::copy(blkw(Gln.data(), l - 1), blkw(Gln.data(), l - 1) + n2, sig.begin());
    w.gemm('n', 'n', H10.data(), sig.data(), B.data());
    w.gemm('n', 'c', B.data(), H10.data(), C.data());
    for (size_t k = 0; k < n2; k++) C[k] += sL(l, k);
    w.gemm('n', 'n', A.data(), C.data(), B.data());
    w.gemm('n', 'c', B.data(), A.data(), Gn.data());
    std::copy(Gn.begin(), Gn.end(), blkw(Gln.data(), l));
    if (o.want_T) {  // g^L_{l,1} = g_l H_{l,l-1} g^L_{l-1,1}
      w.gemm('n', 'n', H10.data(), GN1.data(), GN1b.data());
      w.gemm('n', 'n', A.data(), GN1b.data(), GN1.data());
    }
  }

  // ---- right contact and G_NN (green_rgf.f90:4031-4066)
  for (size_t k = 0; k < n2; k++) H00[k] = blk(Hii, nx)[k] + sR(nx, k);
  std::copy(blk(H1i, nx), blk(H1i, nx) + n2, H10.begin());
  st->sancho_iters_right = sancho(w, o, E, cms ? blk(Sii, nx) : nullptr, H00.data(), H10.data(),
                                  G00.data(), GBB.data());
  w.gemm('c', 'n', H10.data(), G00.data(), A.data());
  w.gemm('n', 'n', A.data(), H10.data(), sigmar.data());
  w.gemm('n', 'n', H10.data(), blkw(Gl.data(), nx - 1), B.data());
  w.gemm('n', 'c', B.data(), H10.data(), C.data());
  for (size_t k = 0; k < n2; k++) C[k] += H00[k] + sigmar[k];
  zS(nx, C.data(), G00.data());
  w.invert(G00.data());
  if (ldos) std::copy(G00.begin(), G00.end(), ldos + (size_t)(nx - 1) * n2);
  std::copy(blkw(Gln.data(), nx - 1), blkw(Gln.data(), nx - 1) + n2, sig.begin());
  w.gemm('n', 'n', H10.data(), sig.data(), B.data());
  w.gemm('n', 'c', B.data(), H10.data(), C.data());
  const R fR = ferm<R>((E - mur) / ((R)o.boltz * templ));  // TEMPl here: trap T2 (green_rgf.f90:4051)
  for (int j = 0; j < nm; j++)
    for (int i = 0; i < nm; i++) {
      const size_t k = i + (size_t)j * nm;
      sig[k] = -(sigmar[k] - std::conj(sigmar[j + (size_t)i * nm])) * fR + C[k] + sL(nx, k);
    }
  w.gemm('n', 'n', G00.data(), sig.data(), B.data());
  w.gemm('n', 'c', B.data(), G00.data(), Gn.data());
  if (ndens) std::copy(Gn.begin(), Gn.end(), ndens + (size_t)(nx - 1) * n2);
  for (int j = 0; j < nm; j++)
    for (int i = 0; i < nm; i++) {
      const size_t k = i + (size_t)j * nm;
      Gp[k] = Gn[k] + (G00[k] - std::conj(G00[j + (size_t)i * nm]));
    }
  if (pdens) std::copy(Gp.begin(), Gp.end(), pdens + (size_t)(nx - 1) * n2);
  for (int j = 0; j < nm; j++)
    for (int i = 0; i < nm; i++) {
      const size_t k = i + (size_t)j * nm;
      A[k] = -(sigmar[k] - std::conj(sigmar[j + (size_t)i * nm])) * fR;
    }
  w.gemm('n', 'n', A.data(), Gp.data(), B.data());
  for (int j = 0; j < nm; j++)
    for (int i = 0; i < nm; i++) {
      const size_t k = i + (size_t)j * nm;
      A[k] = -(sigmar[k] - std::conj(sigmar[j + (size_t)i * nm])) * (fR - 1.0);
    }
  w.gemm('n', 'n', A.data(), Gn.data(), C.data());
  {
    R tim = 0;
    for (int i = 0; i < nm; i++) tim = tim - (B[i + (size_t)i * nm] - C[i + (size_t)i * nm]).real();
    if (tr) *tr = (double)tim;
  }
  // Caroli T(E): G_{N1} = G_NN H_{N,N-1} g^L_{N-1,1};  T = Re Tr[Gamma_R G_{N1} Gamma_L G_{N1}^H]
  if (o.want_T && T_out) {
    std::vector<cd> gL(n2), gR(n2), X(n2), Y(n2);
    for (int j = 0; j < nm; j++)
      for (int i = 0; i < nm; i++) {
        const size_t k = i + (size_t)j * nm, kt = j + (size_t)i * nm;
        gL[k] = cd(0, 1) * (sigmal[k] - std::conj(sigmal[kt]));
        gR[k] = cd(0, 1) * (sigmar[k] - std::conj(sigmar[kt]));
      }
    w.gemm('n', 'n', H10.data(), GN1.data(), GN1b.data());
    w.gemm('n', 'n', G00.data(), GN1b.data(), X.data());   // X = G_{N1}
    w.gemm('n', 'n', gR.data(), X.data(), Y.data());       // Y = Gamma_R G_{N1}
    w.gemm('n', 'c', gL.data(), X.data(), GN1b.data());    // Gamma_L G_{N1}^H
    R t = 0;
    for (int i = 0; i < nm; i++)
      for (int k = 0; k < nm; k++) t += (Y[i + (size_t)k * nm] * GN1b[k + (size_t)i * nm]).real();
    *T_out = (double)t;
  }

  // ---- backward sweep (green_rgf.f90:4069-4149)
  for (int l = nx - 1; l >= 1; l--) {
    const cd* Hb = H1b(l);
    std::copy(Hb, Hb + n2, H10.begin());
    const cd* Gll = blk(Gl.data(), l);
    const cd* Glnl = blk(Gln.data(), l);
    A = Gn;
    w.gemm('n', 'c', H10.data(), Gll, B.data());
    w.gemm('n', 'n', A.data(), B.data(), C.data());
    std::copy(Glnl, Glnl + n2, A.begin());
    w.gemm('n', 'n', H10.data(), A.data(), B.data());
    w.gemm('n', 'n', G00.data(), B.data(), A.data());
    for (size_t k = 0; k < n2; k++) B[k] = C[k] + A[k];
    w.gemm('c', 'n', H10.data(), B.data(), A.data());  // G<_{l+1,l}
    if (cur)
      for (size_t k = 0; k < n2; k++) cur[(size_t)(l - 1) * n2 + k] = A[k].real();
    A = Gn;
    w.gemm('n', 'c', Gll, H10.data(), B.data());
    w.gemm('n', 'n', B.data(), A.data(), C.data());
    std::copy(Glnl, Glnl + n2, A.begin());
    w.gemm('n', 'c', A.data(), H10.data(), B.data());
    w.gemm('n', 'c', B.data(), G00.data(), A.data());
    for (size_t k = 0; k < n2; k++) B[k] = C[k] + A[k];
    if (GLi1) std::copy(B.begin(), B.end(), GLi1 + (size_t)(l - 1) * n2);
    w.gemm('n', 'n', H10.data(), B.data(), A.data());  // G<_{l,l+1}
    if (cur)
      for (size_t k = 0; k < n2; k++) cur[(size_t)(l - 1) * n2 + k] -= A[k].real();
    if (GGi1) {
      // Reproduces the reference: Glp is never filled (zero); in RS Gp keeps
      // its value from the right closure (green_rgf.f90:4094-4103, trap T4),
      // in CMS it is the running G^> of block l+1 (:4313-4322).
      A = Gp;
      w.gemm('c', 'c', Gll, H10.data(), B.data());
      w.gemm('n', 'n', B.data(), A.data(), C.data());
      std::fill(A.begin(), A.end(), cd(0, 0));
      w.gemm('n', 'c', A.data(), H10.data(), B.data());
      w.gemm('n', 'n', B.data(), G00.data(), A.data());
      for (size_t k = 0; k < n2; k++) B[k] = C[k] + A[k];
      std::copy(B.begin(), B.end(), GGi1 + (size_t)(l - 1) * n2);
    }
    std::copy(Gll, Gll + n2, D.begin());
    w.gemm('n', 'c', D.data(), H10.data(), B.data());
    w.gemm('n', 'n', B.data(), G00.data(), GN0.data());  // G_{l,l+1}
    if (GRi1) std::copy(GN0.begin(), GN0.end(), GRi1 + (size_t)(l - 1) * n2);
    w.gemm('n', 'n', GN0.data(), H10.data(), A.data());
    w.gemm('n', 'n', A.data(), D.data(), C.data());
    for (size_t k = 0; k < n2; k++) G00[k] = Gll[k] + C[k];  // G_{l,l}
    if (ldos) std::copy(G00.begin(), G00.end(), ldos + (size_t)(l - 1) * n2);
    A = Gn;
    w.gemm('n', 'c', D.data(), H10.data(), B.data());
    w.gemm('n', 'n', B.data(), A.data(), C.data());
    w.gemm('n', 'n', C.data(), H10.data(), A.data());
    w.gemm('n', 'c', A.data(), D.data(), C.data());
    for (size_t k = 0; k < n2; k++) Gn[k] = Glnl[k] + C[k];
    std::copy(Glnl, Glnl + n2, A.begin());
    w.gemm('n', 'n', GN0.data(), H10.data(), B.data());
    w.gemm('n', 'n', B.data(), A.data(), C.data());
    for (size_t k = 0; k < n2; k++) Gn[k] += C[k];
    w.gemm('n', 'c', A.data(), H10.data(), B.data());
    w.gemm('n', 'c', B.data(), GN0.data(), C.data());
    for (size_t k = 0; k < n2; k++) Gn[k] += C[k];  // G<_{l,l}
    if (ndens) std::copy(Gn.begin(), Gn.end(), ndens + (size_t)(l - 1) * n2);
    if (cms) {
      // CMS recurses G^> like G^< with the never-filled Glp (zero):
      // Gp = Glp + g H10^H Gp H10 g^H + GN0 H10 Glp + Glp H10^H GN0^H  (:4353-4369)
      A = Gp;
      w.gemm('n', 'c', D.data(), H10.data(), B.data());
      w.gemm('n', 'n', B.data(), A.data(), C.data());
      w.gemm('n', 'n', C.data(), H10.data(), A.data());
      w.gemm('n', 'c', A.data(), D.data(), C.data());
      Gp = C;
      if (pdens) std::copy(Gp.begin(), Gp.end(), pdens + (size_t)(l - 1) * n2);
    } else if (pdens)
      for (int j = 0; j < nm; j++)
        for (int i = 0; i < nm; i++) {
          const size_t k = i + (size_t)j * nm;
          pdens[(size_t)(l - 1) * n2 + k] = Gn[k] + (G00[k] - std::conj(G00[j + (size_t)i * nm]));
        }
  }

  // ---- left trace (green_rgf.f90:4151-4160); TEMPr here: trap T2
  for (int j = 0; j < nm; j++)
    for (int i = 0; i < nm; i++) {
      const size_t k = i + (size_t)j * nm;
      Gp[k] = Gn[k] + (G00[k] - std::conj(G00[j + (size_t)i * nm]));
    }
  const R fL = ferm<R>((E - mul) / ((R)o.boltz * tempr));
  for (int j = 0; j < nm; j++)
    for (int i = 0; i < nm; i++) {
      const size_t k = i + (size_t)j * nm;
      A[k] = -(sigmal[k] - std::conj(sigmal[j + (size_t)i * nm])) * fL;
    }
  w.gemm('n', 'n', A.data(), Gp.data(), B.data());
  for (int j = 0; j < nm; j++)
    for (int i = 0; i < nm; i++) {
      const size_t k = i + (size_t)j * nm;
      A[k] = -(sigmal[k] - std::conj(sigmal[j + (size_t)i * nm])) * (fL - 1.0);
    }
  w.gemm('n', 'n', A.data(), Gn.data(), C.data());
  {
    R tim = 0;
    for (int i = 0; i < nm; i++) tim = tim + (B[i + (size_t)i * nm] - C[i + (size_t)i * nm]).real();
    if (tre) *tre = (double)tim;
  }
  auto back = [&](const std::vector<cd>& v, cdd* p) {
    if (p)
      for (size_t k = 0; k < nall; k++) p[k] = cdd((double)v[k].real(), (double)v[k].imag());
  };
  back(nd_v, ndens_out);
  back(pd_v, pdens_out);
  back(ld_v, ldos_out);
  back(gr_v, GRi1_out);
  back(gl_v, GLi1_out);
  back(gg_v, GGi1_out);
  if (cur_out)
    for (size_t k = 0; k < nall; k++) cur_out[k] = (double)cur_v[k];
  return st->status;
}

}  // namespace

extern "C" int oracle_rgf_energy(const OracleOpts* opts, int64_t nm64, int64_t nx64, double E,
                                 const double* mu, const double* temp, const cd* Sii, const cd* Hii,
                                 const cd* H1i, const cd* sig_lesser, const cd* sig_r,
                                 cd* ndens, cd* pdens, cd* ldos, double* tr, double* tre,
                                 double* cur, cd* GRi1, cd* GLi1, cd* GGi1, double* T_out,
                                 OracleStat* st) {
  return rgf_energy<double>(opts, nm64, nx64, E, mu, temp, Sii, Hii, H1i, sig_lesser, sig_r, ndens,
                            pdens, ldos, tr, tre, cur, GRi1, GLi1, GGi1, T_out, st);
}

// The same computation in x87 extended precision (64-bit mantissa) with
// plain loops: the ground truth that FP64 results are measured against.
extern "C" int oracle_rgf_energy_ld(const OracleOpts* opts, int64_t nm64, int64_t nx64, double E,
                                    const double* mu, const double* temp, const cd* Sii, const cd* Hii,
                                    const cd* H1i, const cd* sig_lesser, const cd* sig_r,
                                    cd* ndens, cd* pdens, cd* ldos, double* tr, double* tre,
                                    double* cur, cd* GRi1, cd* GLi1, cd* GGi1, double* T_out,
                                    OracleStat* st) {
  return rgf_energy<long double>(opts, nm64, nx64, E, mu, temp, Sii, Hii, H1i, sig_lesser, sig_r,
                                 ndens, pdens, ldos, tr, tre, cur, GRi1, GLi1, GGi1, T_out, st);
}

// Batch over energy points, one worker thread per core and one energy per
// call, mirroring `!$omp parallel do ie` around green_RGF_RS
// (green_rgf.f90:2916-2925) with single-threaded BLAS.  Hii/H1i are shared by
// all points; per-point arrays are strided by nm*nm*nx elements (cur by the
// same count of doubles).  Null arrays are skipped.  Sii non-null runs
// green_RGF_CMS instead of green_RGF_RS.
extern "C" int oracle_rgf_batch(const OracleOpts* opts, int64_t nm, int64_t nx, int64_t nE,
                                const double* E, const double* mu, const double* temp,
                                const cd* Sii, const cd* Hii, const cd* H1i, const cd* sig_lesser,
                                const cd* sig_r, cd* ndens, cd* pdens, cd* ldos, double* tr,
                                double* tre, double* cur, cd* GRi1, cd* GLi1, cd* GGi1,
                                double* T_out, OracleStat* stats, int n_threads, int extended) {
  const size_t per = (size_t)nm * nm * nx;
  std::atomic<int64_t> next(0);
  std::atomic<int> worst(0);
  auto worker = [&]() {
    for (;;) {
      const int64_t e = next.fetch_add(1);
      if (e >= nE) break;
      OracleStat st{};
      const int s = (extended ? oracle_rgf_energy_ld : oracle_rgf_energy)(
          opts, nm, nx, E[e], mu, temp, Sii, Hii, H1i, sig_lesser ? sig_lesser + e * per : nullptr,
          sig_r ? sig_r + e * per : nullptr, ndens ? ndens + e * per : nullptr,
          pdens ? pdens + e * per : nullptr, ldos ? ldos + e * per : nullptr,
          tr ? tr + e : nullptr, tre ? tre + e : nullptr, cur ? cur + e * per : nullptr,
          GRi1 ? GRi1 + e * per : nullptr, GLi1 ? GLi1 + e * per : nullptr,
          GGi1 ? GGi1 + e * per : nullptr, T_out ? T_out + e : nullptr, &st);
      if (stats) stats[e] = st;
      int cur_w = worst.load();
      while ((s | cur_w) != cur_w && !worst.compare_exchange_weak(cur_w, s | cur_w)) {}
    }
  };
  if (n_threads < 1) n_threads = 1;
  std::vector<std::thread> pool;
  for (int t = 1; t < n_threads; t++) pool.emplace_back(worker);
  worker();
  for (auto& t : pool) t.join();
  return worst.load();
}

// ---------------------------------------------------------------- RGF_W
// green_rgf_calc_w (green_rgf.f90:3399-3831) == RGF_W (rgf_mod.f90:242-674)
// with NBC = 0 and the off-diagonal P blocks absent, as at every call site
// (green_rgf.f90:846, :1551, :3008).  W^R = (I - V P^R)^-1 V by a
// right-to-left sweep of left-connected blocks and a left-to-right sweep;
// W^< / W^> from WR and the imaginary part of the off-diagonal blocks
// (:3803-3829), with the routine's transposes and index max(ix-1,1) as they
// are.  The routine's LL / LG blocks (:3495-3560), its wln / wlp (:3702-3708)
// and its XR recursion (:3752-3757) feed nothing that is returned and are not
// restated.  WRi1 (if non-null) receives blocks 1..nx-1 of the full complex
// off-diagonal block; block nx is left untouched.
namespace {

template <typename R>
int rgf_w_energy(int64_t nm64, int64_t nx64, const cd* Vii_in, const cd* V1i_in, const cd* PL_in,
                 const cd* PG_in, const cd* PR_in, cd* WL_out, cd* WG_out, cd* WR_out, cd* WRi1_out,
                 OracleStat* st) {
  typedef std::complex<R> C;
  typedef std::complex<double> cdd;
  OracleStat dummy{};
  if (!st) st = &dummy;
  std::memset(st, 0, sizeof(*st));
  if (nm64 < 1 || nx64 < 2 || nm64 > 4096) { st->status = ST_BAD_ARGS; return ST_BAD_ARGS; }
  const int nm = (int)nm64, nx = (int)nx64;
  const size_t n2 = nn(nm), nall = n2 * (size_t)nx;
  Work<R> w(nm, st);
  std::vector<C> Vii(Vii_in, Vii_in + nall), V1i(V1i_in, V1i_in + nall), PL(PL_in, PL_in + nall),
      PG(PG_in, PG_in + nall), PR(PR_in, PR_in + nall);
  auto b = [&](std::vector<C>& v, int l) { return v.data() + (size_t)(l - 1) * n2; };  // 1-based
  std::vector<C> M(nall), M1i(nall), Mi1(nall), xlr(nall), Wlr(nall), WR(nall), WRi1(nall);
  std::vector<C> A(n2), B(n2), Cm(n2), D(n2), T1(n2);
  // S = V P^R; M = I - S, M1i = -S_{i+1,i}, Mi1 = -S_{i,i+1} (:3450-3485)
  for (int ix = 1; ix <= nx; ix++) {
    w.gemm('n', 'n', b(Vii, ix), b(PR, ix), A.data());
    for (size_t k = 0; k < n2; k++) b(M, ix)[k] = -A[k];
    for (int i = 0; i < nm; i++) b(M, ix)[i + (size_t)i * nm] += C(1, 0);
  }
  for (int i = 1; i <= nx - 1; i++) {
    w.gemm('n', 'n', b(V1i, i), b(PR, i), A.data());
    for (size_t k = 0; k < n2; k++) b(M1i, i)[k] = -A[k];
    w.gemm('c', 'n', b(V1i, i), b(PR, i + 1), A.data());
    for (size_t k = 0; k < n2; k++) b(Mi1, i)[k] = -A[k];
  }
  std::copy(b(M1i, nx - 1), b(M1i, nx - 1) + n2, b(M1i, nx));
  std::copy(b(Mi1, nx - 1), b(Mi1, nx - 1) + n2, b(Mi1, nx));
  // right-to-left pass (:3710-3722)
  std::copy(b(M, nx), b(M, nx) + n2, A.begin());
  w.invert(A.data());
  std::copy(A.begin(), A.end(), b(xlr, nx));
  w.gemm('n', 'n', A.data(), b(Vii, nx), b(Wlr, nx));
  for (int ix = nx - 1; ix >= 1; ix--) {
    w.gemm('n', 'n', b(Mi1, ix), b(xlr, ix + 1), B.data());
    w.gemm('n', 'n', B.data(), b(M1i, ix), Cm.data());
    for (size_t k = 0; k < n2; k++) A[k] = b(M, ix)[k] - Cm[k];
    w.invert(A.data());
    std::copy(A.begin(), A.end(), b(xlr, ix));
    w.gemm('n', 'n', B.data(), b(V1i, ix), Cm.data());
    for (size_t k = 0; k < n2; k++) D[k] = b(Vii, ix)[k] - Cm[k];
    w.gemm('n', 'n', A.data(), D.data(), b(Wlr, ix));
  }
  // left-to-right pass (:3740-3778)
  auto offdiag = [&](int ix) {  // WRi1_(ix) = (V1i(ix)^T - WR(ix) M1i(ix)^T) xlr(ix+1)^T
    w.gemm('n', 't', b(WR, ix), b(M1i, ix), B.data());
    for (int j = 0; j < nm; j++)
      for (int i = 0; i < nm; i++) Cm[i + (size_t)j * nm] = b(V1i, ix)[j + (size_t)i * nm] - B[i + (size_t)j * nm];
    w.gemm('n', 't', Cm.data(), b(xlr, ix + 1), b(WRi1, ix));
  };
  std::copy(b(Wlr, 1), b(Wlr, 1) + n2, b(WR, 1));
  offdiag(1);
  for (int ix = 2; ix <= nx; ix++) {
    w.gemm('n', 'n', b(xlr, ix), b(M1i, ix - 1), B.data());
    w.gemm('n', 'n', B.data(), b(WRi1, ix - 1), Cm.data());
    for (size_t k = 0; k < n2; k++) b(WR, ix)[k] = b(Wlr, ix)[k] - Cm[k];
    if (ix < nx) offdiag(ix);
  }
  if (WRi1_out)
    for (size_t k = 0; k < n2 * (size_t)(nx - 1); k++)
      WRi1_out[k] = cdd((double)WRi1[k].real(), (double)WRi1[k].imag());
  // W^< and W^> (:3786-3829): the off-diagonal blocks enter with their real
  // part zeroed
  for (size_t k = 0; k < nall; k++) WRi1[k] = C(R(0) * WRi1[k].real(), WRi1[k].imag());
  auto wlg = [&](std::vector<C>& P, cd* out) {
    for (int ix = 1; ix <= nx; ix++) {
      w.gemm('n', 'n', b(WR, ix), b(P, ix), A.data());
      w.gemm('n', 'c', A.data(), b(WR, ix), B.data());
      const int jo = ix < nx ? ix : ix - 1, jp = ix < nx ? ix + 1 : nx;
      for (size_t k = 0; k < n2; k++) T1[k] = -b(WRi1, jo)[k];
      w.gemm('n', 'n', b(WRi1, jo), b(P, jp), A.data());
      w.gemm('n', 't', A.data(), T1.data(), Cm.data());
      for (size_t k = 0; k < n2; k++) B[k] += Cm[k];
      const int m = ix - 1 > 1 ? ix - 1 : 1;
      for (size_t k = 0; k < n2; k++) T1[k] = -b(WRi1, m)[k];
      w.gemm('t', 'n', b(WRi1, m), b(P, m), A.data());
      w.gemm('n', 'n', A.data(), T1.data(), Cm.data());
      for (size_t k = 0; k < n2; k++) B[k] += Cm[k];
      if (out)
        for (size_t k = 0; k < n2; k++)
          out[(size_t)(ix - 1) * n2 + k] = cdd((double)B[k].real(), (double)B[k].imag());
    }
  };
  wlg(PL, WL_out);
  wlg(PG, WG_out);
  if (WR_out)
    for (size_t k = 0; k < nall; k++) WR_out[k] = cdd((double)WR[k].real(), (double)WR[k].imag());
  return st->status;
}

}  // namespace

// Batch of W solves: one device (Vii, V1i) and nE polarization sets
// (PL, PG, PR strided by nm*nm*nx), one per worker thread.
extern "C" int oracle_rgf_w_batch(int64_t nm, int64_t nx, int64_t nE, const cd* Vii, const cd* V1i,
                                  const cd* PL, const cd* PG, const cd* PR, cd* WL, cd* WG, cd* WR,
                                  cd* WRi1, OracleStat* stats, int n_threads, int extended) {
  const size_t per = (size_t)nm * nm * nx;
  std::atomic<int64_t> next(0);
  std::atomic<int> worst(0);
  auto worker = [&]() {
    for (;;) {
      const int64_t e = next.fetch_add(1);
      if (e >= nE) break;
      OracleStat st{};
      auto off = [&](cd* p) { return p ? p + e * per : nullptr; };
      const int s = extended
          ? rgf_w_energy<long double>(nm, nx, Vii, V1i, PL + e * per, PG + e * per, PR + e * per,
                                      off(WL), off(WG), off(WR), off(WRi1), &st)
          : rgf_w_energy<double>(nm, nx, Vii, V1i, PL + e * per, PG + e * per, PR + e * per, off(WL),
                                 off(WG), off(WR), off(WRi1), &st);
      if (stats) stats[e] = st;
      int cur_w = worst.load();
      while ((s | cur_w) != cur_w && !worst.compare_exchange_weak(cur_w, s | cur_w)) {}
    }
  };
  if (n_threads < 1) n_threads = 1;
  std::vector<std::thread> pool;
  for (int t = 1; t < n_threads; t++) pool.emplace_back(worker);
  worker();
  for (auto& t : pool) t.join();
  return worst.load();
}

// ---------------------------------------------------------- GW convolutions
// The polarization and GW self-energy of green_rgf_solve_gw_3d
// (green_rgf.f90:2944-3092): banded (|i-j| <= ndiag) direct energy / k sums,
// accumulated in the reference's loop order per element.  All arrays are
// (nm,nm,nx,nen,nk) column-major; nk = nky*nkz, ik = ikz + (iky-1)*nkz.
// imag_only: read G with its real part zeroed (the reference zeroes it in
// place before P, :2940-2942, and Sigma then sees the same arrays).
namespace {

const double kPiGW = 3.14159265359;  // the module's pi (green_rgf.f90:23)

struct GWIdx {
  int64_t nm, nx, nen, nky, nkz;
  size_t at(int64_t i, int64_t j, int64_t ix, int64_t ie, int64_t ik) const {  // 1-based
    return (size_t)(i - 1) + (size_t)nm * ((j - 1) + (size_t)nm * ((ix - 1) + (size_t)nx * ((ie - 1) + (size_t)nen * (ik - 1))));
  }
  int64_t kd(int64_t iky, int64_t ikz, int64_t iqy, int64_t iqz) const {  // :2968-2977
    int64_t ikzd = ikz - iqz + nkz / 2, ikyd = iky - iqy + nky / 2;
    if (ikzd < 1) ikzd += nkz;
    if (ikzd > nkz) ikzd -= nkz;
    if (ikyd < 1) ikyd += nky;
    if (ikyd > nky) ikyd -= nky;
    if (nky == 1) ikyd = 1;
    if (nkz == 1) ikzd = 1;
    return ikzd + (ikyd - 1) * nkz;
  }
};

inline cd gread(const cd* G, size_t k, int imag_only) {
  return imag_only ? cd(0.0 * G[k].real(), G[k].imag()) : G[k];
}

}  // namespace

extern "C" void oracle_gw_polarization(int64_t nm, int64_t nx, int64_t nen, int64_t nky, int64_t nkz,
                                       int64_t ndiag, double dEn, double spindeg, int imag_only,
                                       const cd* GL, const cd* GG, const cd* GR, cd* PL, cd* PG,
                                       cd* PR, int n_threads) {
  const GWIdx X{nm, nx, nen, nky, nkz};
  const int64_t nk = nky * nkz, nopmax = nen / 2 - 10;
  const size_t total = (size_t)nm * nm * nx * nen * nk;
  std::fill(PL, PL + total, cd(0, 0));
  std::fill(PG, PG + total, cd(0, 0));
  std::fill(PR, PR + total, cd(0, 0));
  std::atomic<int64_t> next(-nopmax);
  auto worker = [&]() {
    for (;;) {
      const int64_t nop = next.fetch_add(1);
      if (nop > nopmax) break;
      const int64_t iop = nop + nen / 2;
      for (int64_t iqy = 1; iqy <= nky; iqy++)
        for (int64_t iqz = 1; iqz <= nkz; iqz++) {
          const int64_t iq = iqz + (iqy - 1) * nkz;
          for (int64_t ix = 1; ix <= nx; ix++)
            for (int64_t i = 1; i <= nm; i++) {
              const int64_t l = std::max<int64_t>(i - ndiag, 1), h = std::min<int64_t>(nm, i + ndiag);
              for (int64_t iky = 1; iky <= nky; iky++)
                for (int64_t ikz = 1; ikz <= nkz; ikz++) {
                  const int64_t ik = ikz + (iky - 1) * nkz, ikd = X.kd(iky, ikz, iqy, iqz);
                  for (int64_t ie = std::max<int64_t>(nop + 1, 1); ie <= std::min<int64_t>(nen, nen + nop); ie++)
                    for (int64_t j = l; j <= h; j++) {
                      const size_t o = X.at(i, j, ix, iop, iq);
                      const size_t a = X.at(i, j, ix, ie, ik), bt = X.at(j, i, ix, ie - nop, ikd),
                                   b = X.at(i, j, ix, ie - nop, ikd);
                      PL[o] += gread(GL, a, imag_only) * gread(GG, bt, imag_only);
                      PG[o] += gread(GG, a, imag_only) * gread(GL, bt, imag_only);
                      PR[o] += gread(GL, a, imag_only) * std::conj(gread(GR, b, imag_only)) +
                               gread(GR, a, imag_only) * gread(GL, bt, imag_only);
                    }
                }
            }
        }
    }
  };
  if (n_threads < 1) n_threads = 1;
  std::vector<std::thread> pool;
  for (int t = 1; t < n_threads; t++) pool.emplace_back(worker);
  worker();
  for (auto& t : pool) t.join();
  const cd dE = cd(0.0, -1.0 * dEn / 2.0 / kPiGW) * spindeg / (double)nk;  // :2996
  for (size_t k = 0; k < total; k++) { PL[k] *= dE; PG[k] *= dE; PR[k] *= dE; }
}

// New self-energies (:3020-3068), then Sigma^R's imaginary part from
// Sigma^> - Sigma^<, symmetrisation, mixing into the *_gw arrays and the
// edge-block copies (:3069-3092).  SL / SG / SR are the *_gw arrays (inout).
extern "C" void oracle_gw_self_energy(int64_t nm, int64_t nx, int64_t nen, int64_t nky, int64_t nkz,
                                      int64_t ndiag, double dEn, double alpha_mix, int imag_only,
                                      const cd* GL, const cd* GG, const cd* GR, const cd* WL,
                                      const cd* WG, const cd* WR, cd* SL, cd* SG, cd* SR,
                                      int n_threads) {
  const GWIdx X{nm, nx, nen, nky, nkz};
  const int64_t nk = nky * nkz, nopmax = nen / 2 - 10;
  const size_t total = (size_t)nm * nm * nx * nen * nk;
  std::vector<cd> nL(total, cd(0, 0)), nG(total, cd(0, 0)), nR(total, cd(0, 0));
  std::atomic<int64_t> next(1);
  auto worker = [&]() {
    for (;;) {
      const int64_t ie = next.fetch_add(1);
      if (ie > nen) break;
      for (int64_t iky = 1; iky <= nky; iky++)
        for (int64_t ikz = 1; ikz <= nkz; ikz++)
          for (int64_t nop = -nopmax; nop <= nopmax; nop++) {
            if (!(ie > std::max<int64_t>(nop, 1) && ie < nen + nop)) continue;
            const int64_t ik = ikz + (iky - 1) * nkz, iop = nop + nen / 2;
            for (int64_t iqy = 1; iqy <= nky; iqy++)
              for (int64_t iqz = 1; iqz <= nkz; iqz++) {
                const int64_t iq = iqz + (iqy - 1) * nkz, ikd = X.kd(iky, ikz, iqy, iqz);
                for (int64_t ix = 1; ix <= nx; ix++)
                  for (int64_t i = 1; i <= nm; i++) {
                    const int64_t l = std::max<int64_t>(i - ndiag, 1), h = std::min<int64_t>(nm, i + ndiag);
                    for (int64_t j = l; j <= h; j++) {
                      const size_t o = X.at(i, j, ix, ie, ik), g = X.at(i, j, ix, ie - nop, ikd),
                                   w = X.at(i, j, ix, iop, iq);
                      nL[o] += gread(GL, g, imag_only) * WL[w];
                      nG[o] += gread(GG, g, imag_only) * WG[w];
                      nR[o] += gread(GL, g, imag_only) * WR[w] + gread(GR, g, imag_only) * WL[w] +
                               gread(GR, g, imag_only) * WR[w];
                    }
                  }
              }
          }
    }
  };
  if (n_threads < 1) n_threads = 1;
  std::vector<std::thread> pool;
  for (int t = 1; t < n_threads; t++) pool.emplace_back(worker);
  worker();
  for (auto& t : pool) t.join();
  const cd dE = cd(0.0, dEn / 2.0 / kPiGW) / (double)nk;  // :3064
  for (size_t k = 0; k < total; k++) {
    nL[k] *= dE;
    nG[k] *= dE;
    nR[k] *= dE;
  }
  for (size_t k = 0; k < total; k++) nR[k] = cd(nR[k].real(), (nG[k] - nL[k]).imag() / 2.0);  // :3068
  const size_t n2 = (size_t)nm * nm;
  std::vector<cd> B(n2);
  for (size_t blk = 0; blk < total / n2; blk++)  // symmetrise each (ix, ie, ik) block (:3070-3081)
    for (std::vector<cd>* A : {&nR, &nL, &nG}) {
      cd* a = A->data() + blk * n2;
      for (int64_t j = 0; j < nm; j++)
        for (int64_t i = 0; i < nm; i++) B[i + j * nm] = a[j + i * nm];
      for (size_t k = 0; k < n2; k++) a[k] = (a[k] + B[k]) / 2.0;
    }
  for (size_t k = 0; k < total; k++) {  // mixing (:3083-3085)
    SR[k] = SR[k] + alpha_mix * (nR[k] - SR[k]);
    SL[k] = SL[k] + alpha_mix * (nL[k] - SL[k]);
    SG[k] = SG[k] + alpha_mix * (nG[k] - SG[k]);
  }
  auto copy_block = [&](cd* A, int64_t dst, int64_t src) {  // A(:,:,dst,:,:) = A(:,:,src,:,:)
    for (int64_t ik = 1; ik <= nk; ik++)
      for (int64_t ie = 1; ie <= nen; ie++)
        std::copy(A + X.at(1, 1, src, ie, ik), A + X.at(1, 1, src, ie, ik) + n2, A + X.at(1, 1, dst, ie, ik));
  };
  for (int64_t ix = 1; ix <= 2; ix++)  // :3087-3091
    for (cd* A : {SR, SL, SG}) copy_block(A, ix, 3);
  for (int64_t ix = 1; ix <= 2; ix++)
    for (cd* A : {SR, SL, SG}) copy_block(A, nx - ix + 1, nx - 2);
}

// calc_n_electron (green_rgf.f90:3920-3945) for one k-point set laid out as
// (nm,nm,nx,nen,nk).  nelec/pelec have nx entries.
extern "C" void oracle_calc_n_electron(const cd* G_lesser, const cd* G_greater, int64_t nen,
                                       const double* E, int64_t nm, int64_t nk, int64_t nx,
                                       double* nelec, double* pelec, const double* midgap) {
  const double pi = 3.14159265359;  // green_rgf.f90:23
  const double dE = (E[1] - E[0]) / (2.0 * pi);
  const double dK = 2.0 * pi / (double)nk;
  const size_t n2 = (size_t)nm * nm;
  for (int64_t ix = 0; ix < nx; ix++) { nelec[ix] = 0.0; pelec[ix] = 0.0; }
  for (int64_t i = 0; i < nen; i++)
    for (int64_t ik = 0; ik < nk; ik++)
      for (int64_t ix = 0; ix < nx; ix++)
        for (int64_t j = 0; j < nm; j++) {
          const size_t off = (size_t)j + (size_t)j * nm + ix * n2 + (size_t)nx * n2 * (i + (size_t)nen * ik);
          if (E[i] > midgap[ix])
            nelec[ix] = nelec[ix] + G_lesser[off].imag() * dE * dK;
          else
            pelec[ix] = pelec[ix] - G_greater[off].imag() * dE * dK;
        }
}

// calc_block_current (green_rgf.f90:4602-4640): bond current between the
// sub-blocks ib, ib+1 (nb orbitals each, ns per block) of every block, per
// energy (jdens) and summed over energies (tot_cur, tot_ecur).  The last
// sub-block of each block repeats the previous sub-block's values, as the
// reference does; for ns = 1 the reference uses an unset matrix there, taken
// as zero here.  H (nm,nm,nx), G_lesser (nm,nm,nx,nen); outputs (nb,nb,nx*ns[,nen]).
extern "C" void oracle_calc_block_current(const cd* H, const cd* G_lesser, int64_t nen,
                                          const double* en, double spindeg, int64_t nb,
                                          int64_t ns, int64_t nm, int64_t nx, double* tot_cur,
                                          double* tot_ecur, double* jdens) {
  const double e0 = 1.6022e-19, hbar = 1.0546e-34, tpi = 6.28318530718;
  const size_t n2 = (size_t)nm * nm, b2 = (size_t)nb * nb, nl = (size_t)nx * ns;
  for (size_t k = 0; k < b2 * nl; k++) { tot_cur[k] = 0.0; if (tot_ecur) tot_ecur[k] = 0.0; }
  std::vector<cd> B(b2, cd(0.0, 0.0));
  const double scale = (en[1] - en[0]) * e0 / tpi / hbar * e0 * spindeg;
  for (int64_t ie = 0; ie < nen; ie++)
    for (int64_t ix = 0; ix < nx; ix++) {
      const cd* Hx = H + ix * n2;
      const cd* Gx = G_lesser + ix * n2 + (size_t)ie * nx * n2;
      if (ns == 1) std::fill(B.begin(), B.end(), cd(0.0, 0.0));
      for (int64_t ib = 1; ib <= ns; ib++) {
        if (ib < ns) {
          for (int64_t io = 0; io < nb; io++)
            for (int64_t jo = 0; jo < nb; jo++) {
              const size_t i = io + (ib - 1) * nb, j = jo + ib * nb;
              const cd b = Hx[i + j * nm] * Gx[j + i * nm] - Hx[j + i * nm] * Gx[i + j * nm];
              B[io + jo * nb] = b * scale;
            }
        }
        const size_t l = (size_t)ix * ns + (ib - 1);
        for (size_t k = 0; k < b2; k++) {
          const double v = B[k].real();
          if (jdens) jdens[k + l * b2 + (size_t)ie * nl * b2] = v;
          if (tot_ecur) tot_ecur[k + l * b2] += en[ie] * v;
          tot_cur[k + l * b2] += v;
        }
      }
    }
}
