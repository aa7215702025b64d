// rgf_solver.cuh -- the per-energy RGF chain of green_RGF_RS as a CTA-wide
// device routine, templated on the block-operation policy (GEMM + inverse
// kernels for a block size).  Each policy is instantiated in its own
// translation unit (rgf_task_*.cu) as one non-inlined task function; the
// persistent kernel in rgf_fp64.cu calls the one matching each task's block
// size, so one launch can drain tasks of any mix of block sizes.
//
// The chain follows the reference routine green_RGF_RS
// (src/green_rgf.f90:3950-4164):
//
//   left lead   Sancho-Rubio (sancho, :4451-4537) and Sigma_L     :3990-4012
//   forward     g_l, g^<_l for l = 2..nx-1                         :4013-4030
//   right lead  Sancho-Rubio, Sigma_R, G_NN, G^<_NN, tr            :4031-4066
//   backward    G_ll, G_{l,l+1}, G^<_ll, G^>_ll, cur(:,:,l)        :4069-4149
//   left trace  tre                                                :4151-4160
//   T(E)        Caroli Tr[Gamma_R G_N1 Gamma_L G_N1^H] (green.f90:2571-2580)
//               from a running left-connected column g^L_{l,1}.
//
// Differences in *how* (not what) it is computed:
//   - products the reference forms twice are formed once, and the
//     reference's H10 Gl^H and (Gl H10^H G< H10) Gl^H reuse Gl H10^H
//     (15 complex products per backward block instead of 22; 9 when
//     neither `cur` nor GLi1 is requested);
//   - without scattering Sigma^<, g^<_l = g^L_{l,1} Sigma^<_L g^L_{l,1}^H
//     = i fL V_l V_l^H with V_l = g^L_{l,1} L, Gamma_L = L L^H (pivoted
//     Cholesky): one product per forward block instead of four, T(E) from
//     V as well; the last backward G^< term is the conjugate transpose of
//     another;
//   - sums, z*I - H - Sigma assembly, Fermi-weighted Sigma^< and the
//     G^> = G^< + G^R - G^A identity are fused into the product epilogues;
//   - the traces tr / tre / T form only the diagonal of the final product;
//   - the dead Sancho GBB inverse (:4527-4529) and the always-zero Glp terms
//     of GGi1 (:4094-4103) are skipped.
// The result is the same function of the inputs up to rounding.
#pragma once
#include <cstdio>
#include <type_traits>

#include "rgf_device.cuh"
#include "rgf_internal.h"
#include "rgf_staged.cuh"
#include "rgf_tasks.h"

namespace rgf {

namespace {


enum TmpBlock {
  T_H00 = 0, T_SA, T_SB, T_HBB, T_HSS, T_H10A, T_H10B, T_H01A, T_H01B, T_GS,
  T_SIGL, T_SIGR, T_SIG, T_F1, T_F2, T_F3, T_F4, T_GN1A, T_GN1B, T_G00A,
  T_G00B, T_GNA, T_GNB, T_Q1, T_Q2, T_Q3, T_Q4, T_R5, T_INV, T_RT,
  T_SRS, T_SLS,  // green_RGF_CMS: sigma_r_ph S_ll, sigma_lesser_ph S_ll of the current block
  T_COUNT,
  T_X3 = T_SLS,  // backward sweep (T_SLS is only live before it)
  // aliases (lifetimes do not overlap)
  T_P2 = T_F2, T_P3 = T_F3, T_P4 = T_SIG,
  T_GPN = T_SB, T_X1 = T_SA, T_X2 = T_H10A, T_Y = T_H10B, T_Z = T_H01A,
  T_GAML = T_H01B, T_GAMR = T_HSS, T_R1 = T_GS,
};
static_assert(T_COUNT <= kNumTemps, "temp blocks");


constexpr int kSmemXMaxNb = 64;  // generic path: inverse workspace in shared memory up to this nb

// Any nb that is a multiple of 8: register-direct DMMA GEMM (warp tiles of
// TM x TN 8x8 subtiles), unblocked Gauss-Jordan.
template <int TM, int TN>
struct GenericOps {
  static constexpr bool kMixed = false;
  static constexpr int kMinBlocks = 2;
  static size_t smem_bytes(int nb) {
    return ((nb <= kSmemXMaxNb ? (size_t)nb * nb : 0) + 2 * (size_t)nb) * sizeof(double2);
  }
  SmemInv& inv;
  double2* X;
  double2* rowk;
  __device__ GenericOps(SmemInv& i, double2* dyn, double2* slot_inv, double2*, int n)
      : inv(i), X(n <= kSmemXMaxNb ? dyn : slot_inv),
        rowk(dyn + (n <= kSmemXMaxNb ? (size_t)n * n : 0)) {}
  template <class Epi>
  __device__ void gemm(int n, const double2* A, bool cA, const double2* B, bool cB, Epi&& epi) {
    cgemm<TM, TN>(n, A, cA, B, cB, epi);
  }
  __device__ int invert(int n, double2* dst, double2* dst2) {
    return gj_invert(n, X, dst, dst2, inv, rowk, rowk + n);
  }
  // >= n complex values of shared memory free between block operations
  __device__ double2* scratch() const { return rowk; }
};

// nb = 32, 64, 128, 256: shared-memory-staged GEMM; inverse in shared memory
// (nb <= 64) or blocked with shared-memory panels.
template <int NB>
struct StagedOps {
  static constexpr bool kMixed = false;
  static constexpr int kMinBlocks = 2;
  static size_t smem_bytes(int) { return StagedCfg<NB>::SMEM; }
  SmemInv& inv;
  double2* dyn;
  double2* X;
  double2* Rt;
  __device__ StagedOps(SmemInv& i, double2* dyn_, double2* slot_inv, double2* slot_rt, int)
      : inv(i), dyn(dyn_), X(StagedCfg<NB>::SMEM_INV ? dyn_ : slot_inv), Rt(slot_rt) {}
  template <class Epi>
  __device__ void gemm(int, const double2* A, bool cA, const double2* B, bool cB, Epi&& epi) {
    gemm_staged<NB>(NB, NB, NB, A, NB, cA, B, NB, cB, dyn, epi);
  }
  __device__ int invert(int, double2* dst, double2* dst2) {
    // nb = 32: matrix in registers (4 elements a thread); nb = 64: in shared
    // memory as one panel of the blocked form (the register form, 16
    // elements a thread, measured slower)
    if constexpr (NB == 32)
      return gj_invert_reg<NB>(X, dst, dst2, inv, dyn + (size_t)NB * NB);
    else if constexpr (StagedCfg<NB>::SMEM_INV)
      return gj_invert_smem_blocked<NB>(X, dst, dst2, inv, dyn + (size_t)NB * NB);
    else return gj_invert_blocked<NB>(X, Rt, dst, dst2, dyn, dyn, inv);
  }
  // >= NB complex values of shared memory free between block operations
  __device__ double2* scratch() const { return dyn; }
};

template <class Ops>
struct Solver {
  KOpts o;
  int64_t nx_max;
  Smem& sm;
  Ops& ops;
  double2* X;       // the matrix to invert is assembled here
  double2* slot;
  int n, nx;
  size_t n2;
  int status = 0, n_gemm = 0, n_inv = 0;

  __device__ Solver(const KOpts& o_, int64_t nx_max_, Smem& sm_, Ops& ops_, double2* slot_,
                    int n_, int nx_)
      : o(o_), nx_max(nx_max_), sm(sm_), ops(ops_), X(ops_.X), slot(slot_), n(n_), nx(nx_),
        n2((size_t)n_ * n_) {}

  __device__ double2* tmp(int k) const { return slot + 2 * nx_max * n2 + (size_t)k * n2; }
  __device__ double2* Gl(int l) const { return slot + (size_t)l * n2; }
  __device__ double2* Gln(int l) const { return slot + (nx_max + l) * n2; }

  // Mixed form only: the block operations of the device chain run in the
  // split-integer / refined form, Sancho-Rubio and its self-energies in FP64.
  __device__ void set_mixed(bool on) {
    if constexpr (Ops::kMixed) ops.mixed_on = on;
  }
  __device__ bool fp64_now() const {
    if constexpr (Ops::kMixed) return !ops.mixed_on;
    return true;
  }

  // n_gemm / n_inv count the products and inverses run in FP64; the mixed
  // form's own operations are counted by its policy.
  template <class Epi>
  __device__ void gemm(const double2* A, bool cA, const double2* B, bool cB, Epi&& epi) {
    if (fp64_now()) n_gemm++;
    ops.gemm(n, A, cA, B, cB, epi);
    __syncthreads();
  }
  // C = op(A) op(B)
  __device__ void gemm_store(const double2* A, bool cA, const double2* B, bool cB, double2* C,
                             double2* C2 = nullptr) {
    const int nn = n;
    gemm(A, cA, B, cB, [&](int i, int j, double2 v) {
      C[i + j * nn] = v;
      if (C2) C2[i + j * nn] = v;
    });
  }
  // X holds the matrix; dst (and dst2) receive its inverse.
  __device__ void invert_X(double2* dst, double2* dst2 = nullptr) {
    if (fp64_now()) n_inv++;
    if (ops.invert(n, dst, dst2)) status |= RGF_ST_SINGULAR;
  }

  // z*S - h for element (i, j): S = I (S == nullptr) or the overlap block S.
  __device__ __forceinline__ static double2 zs_minus(double2 z, const double2* S, int i, int j,
                                                     int idx, double2 h) {
    if (S) return csub(cmul(z, S[idx]), h);
    return (i == j) ? make_double2(z.x - h.x, z.y - h.y) : make_double2(-h.x, -h.y);
  }

  // Cholesky factor of the Hermitian positive semidefinite block G
  // (destroyed): L with G = L L^H, L in G's own row order (diagonal pivoting
  // without interchanges: step k takes the largest remaining diagonal entry
  // as the pivot row, so L is a row permutation of a lower-triangular
  // factor), columns beyond the rank zero.  The pivoted Cholesky
  // factorization of LAPACK's xPSTRF, right-looking, with its default stop:
  // the largest remaining diagonal entry <= n eps times the largest initial
  // one.  Thread i < n owns row i's diagonal and flags.
  // Returns false when G is not positive semidefinite to rounding: a row
  // left out of the factor keeps a remaining diagonal entry below
  // -n eps max_i |G_ii| (an indefinite Gamma, e.g. from a non-retarded
  // sigma or an unconverged lead); L is then unusable and the caller takes
  // the general form.
  __device__ bool chol_psd(double2* G, double2* L) {
    const int nn = n, tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    double2* lcol = ops.scratch();
    const bool own = tid < nn;
    double d = own ? G[tid + tid * nn].x : 0.0;
    bool used = !own;
    double dtol = 0.0;
    double amax = fabs(d);
#pragma unroll
    for (int o = 16; o; o >>= 1) amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
    if (lane == 0) sm.red.v[warp] = amax;
    __syncthreads();
    amax = 0.0;
#pragma unroll
    for (int w = 0; w < kWarps; w++) amax = fmax(amax, sm.red.v[w]);
    __syncthreads();
    const double neg_tol = (double)nn * 2.220446049250313e-16 * amax;
    int k = 0;
    for (; k < nn; k++) {
      unsigned key = 0u;
      if (!used) key = d > 0.0 ? (unsigned)((unsigned long long)__double_as_longlong(d) >> 32) + 2u : 1u;
      const unsigned kmax = __reduce_max_sync(0xffffffffu, key);
      const unsigned imin = __reduce_min_sync(0xffffffffu, key == kmax ? (unsigned)tid : 0xffffffffu);
      if ((unsigned)tid == imin) {
        sm.red.v[warp] = __longlong_as_double((long long)(((unsigned long long)kmax << 32) | imin));
        sm.red.v[kWarps + warp] = d;
      }
      __syncthreads();
      unsigned long long best = (unsigned long long)__double_as_longlong(sm.red.v[0]);
      double dp = sm.red.v[kWarps];
#pragma unroll
      for (int w = 1; w < kWarps; w++) {
        const unsigned long long e = (unsigned long long)__double_as_longlong(sm.red.v[w]);
        const unsigned ek = (unsigned)(e >> 32), bk = (unsigned)(best >> 32);
        if (ek > bk || (ek == bk && (unsigned)e < (unsigned)best)) { best = e; dp = sm.red.v[kWarps + w]; }
      }
      const unsigned bkey = (unsigned)(best >> 32);
      const int p = (int)(unsigned)best;
      if (k == 0) dtol = (double)nn * 2.220446049250313e-16 * dp;
      if (bkey <= 1u || dp <= dtol) break;  // uniform: rank k
      const double s = sqrt(dp), rs = 1.0 / s;
      if (own) {
        double2 l = czero();
        if (tid == p) {
          l = make_double2(s, 0.0);
          used = true;
        } else if (!used) {
          const double2 g = G[tid + p * nn];
          l = make_double2(g.x * rs, g.y * rs);
          d -= l.x * l.x + l.y * l.y;
        }
        L[tid + k * nn] = l;
        lcol[tid] = tid == p ? czero() : l;  // row and column p are never read again
      }
      __syncthreads();
      for_each_elem(n, [&](int i, int j, int idx) {
        const double2 a = lcol[i], b = lcol[j];
        if ((a.x == 0.0 && a.y == 0.0) || (b.x == 0.0 && b.y == 0.0)) return;
        G[idx] = csub(G[idx], cmul(a, cconj(b)));
      });
      __syncthreads();
    }
    for (int e = tid; e < (nn - k) * nn; e += kThreads) L[(size_t)k * nn + e] = czero();
    double dmin = (own && !used) ? d : 0.0;
#pragma unroll
    for (int o = 16; o; o >>= 1) dmin = fmin(dmin, __shfl_xor_sync(0xffffffffu, dmin, o));
    if (lane == 0) sm.red.v[warp] = dmin;
    __syncthreads();
    dmin = 0.0;
#pragma unroll
    for (int w = 0; w < kWarps; w++) dmin = fmin(dmin, sm.red.v[w]);
    __syncthreads();
    return !(dmin < -neg_tol);
  }

  // sancho (green_rgf.f90:4451-4537); S00 = nullptr is the identity (the
  // green_RGF_RS call sites), green_RGF_CMS passes its end blocks' overlap.
  // H00 is a slot block; the coupling argument is H10arg = conj_src ? src^H :
  // src.  Result -> GS.
  __device__ int sancho(double E, const double2* H00, const double2* src, bool conj_src,
                        double2* GS, const double2* S00 = nullptr) {
    const int nn = n;
    const double2 z = make_double2(E, o.eta_lead);
    double2 *H10 = tmp(T_H10A), *H10n = tmp(T_H10B), *H01 = tmp(T_H01A), *H01n = tmp(T_H01B);
    double2 *HBB = tmp(T_HBB), *HSS = tmp(T_HSS), *SA = tmp(T_SA), *SB = tmp(T_SB);
    for_each_elem(n, [&](int i, int j, int idx) {
      HBB[idx] = H00[idx];
      HSS[idx] = H00[idx];
      const double2 a = src[idx], at = src[j + i * nn];
      H10[idx] = conj_src ? cconj(at) : a;
      H01[idx] = conj_src ? a : cconj(at);
    });
    __syncthreads();
    int taken = 0;
    for (int it = 1; it <= o.sancho_nmax; it++) {
      taken = it;
      // A = inv(z*S00 - H_BB)
      for_each_elem(n, [&](int i, int j, int idx) { X[idx] = zs_minus(z, S00, i, j, idx, HBB[idx]); });
      __syncthreads();
      invert_X(SA);
      gemm_store(SA, false, H10, false, SB);                         // B = A H_10
      gemm(H01, false, SB, false, [&](int i, int j, double2 v) {     // C = H_01 B; H_SS += C; H_BB += C
        const int idx = i + j * nn;
        HSS[idx] = cadd(HSS[idx], v);
        HBB[idx] = cadd(HBB[idx], v);
      });
      gemm_store(H10, false, SB, false, H10n);                       // C = H_10 B  (new H_10)
      gemm_store(SA, false, H01, false, SB);                         // B = A H_01
      gemm(H10, false, SB, false, [&](int i, int j, double2 v) {     // A = H_10 B; H_BB += A
        const int idx = i + j * nn;
        HBB[idx] = cadd(HBB[idx], v);
      });
      double err_local = 0.0;
      gemm(H01, false, SB, false, [&](int i, int j, double2 v) {     // C = H_01 B  (new H_01)
        H01n[i + j * nn] = v;
        err_local += sqrt(v.y * v.y + v.x * v.x);
      });
      double2* t1 = H10; H10 = H10n; H10n = t1;
      double2* t2 = H01; H01 = H01n; H01n = t2;
      const double err = block_sum2(make_double2(err_local, 0.0), sm.red).x;
      if (fabs(err) < o.sancho_tol) break;
      if (it == o.sancho_nmax) {
        for_each_elem(n, [&](int, int, int idx) { HSS[idx] = H00[idx]; HBB[idx] = H00[idx]; });
        __syncthreads();
        status |= RGF_ST_SANCHO_NC;
        taken = o.sancho_nmax + 1;
      }
    }
    // G00 = inv(z*S00 - H_SS); the reference's GBB inverse is unused and skipped
    for_each_elem(n, [&](int i, int j, int idx) { X[idx] = zs_minus(z, S00, i, j, idx, HSS[idx]); });
    __syncthreads();
    invert_X(GS);
    return taken;
  }

  // Publishes that the outputs of the last `count` blocks are in memory for
  // a reader outside the GPU (the pipelined host copies): every thread's
  // stores are made visible system-wide, then one thread sets the counter.
  __device__ static void publish(int32_t* progress, int count) {
    if (!progress) return;
    __threadfence_system();
    __syncthreads();
    if (threadIdx.x == 0) *(volatile int32_t*)progress = count;
  }

  __device__ void run(const DTask& tk, const DDev& dv, DInfo* info, int32_t* progress = nullptr) {
    const int nn = n;
    const double E = tk.E;
    const double2 z = make_double2(E, o.eta_dev);
    const double mul = dv.mu[0], mur = dv.mu[1], templ = dv.temp[0], tempr = dv.temp[1];
    const double2* Hii = dv.Hii;
    const double2* H1i = dv.H1i;
    const double2* sl = tk.sig_lesser;
    const double2* sr = tk.sig_r;
    const bool ballistic = sl == nullptr;                          // no scattering Sigma^<
    auto blk = [&](const double2* base, int l) { return base + (size_t)l * n2; };
    auto wblk = [&](double2* base, int l) { return base + (size_t)l * n2; };
    const bool want_T = o.want_T && tk.T;
    // green_RGF_CMS (overlap given): z*S_ll, and the scattering self-energies
    // enter as sigma_r_ph(l) S_ll and sigma_lesser_ph(l) S_ll (:4203-4211,
    // :4225-4240, :4258-4265); green_RGF_RS adds them as they are.
    const double2* Sii = dv.Sii;
    const bool cms = Sii != nullptr;
    auto S_l = [&](int l) -> const double2* { return cms ? blk(Sii, l) : nullptr; };
    auto scat = [&](const double2* sg, int l, int slot) -> const double2* {
      if (!sg) return nullptr;
      if (!cms) return blk(sg, l);
      gemm_store(blk(sg, l), false, blk(Sii, l), false, tmp(slot));
      return tmp(slot);
    };

    // ------------------------------------------------ left contact
    double2* H00 = tmp(T_H00);
    {
      const double2* sr0 = scat(sr, 0, T_SRS);
      for_each_elem(n, [&](int, int, int idx) {
        H00[idx] = sr0 ? cadd(Hii[idx], sr0[idx]) : Hii[idx];
      });
      __syncthreads();
    }
    const double2* H10 = blk(H1i, 0);
    const int itL = sancho(E, H00, H10, true, tmp(T_GS), S_l(0));
    double2* sigmal = tmp(T_SIGL);
    gemm_store(H10, false, tmp(T_GS), false, tmp(T_F1));            // A = H10 G00
    gemm_store(tmp(T_F1), false, H10, true, sigmal);                // sigmal = A H10^H
    const double fl = fermi((E - mul) / (o.boltz * templ));
    {
      double2* sig = tmp(T_SIG);
      double2* gam = tmp(T_F3);
      const double2* sl0 = scat(sl, 0, T_SLS);
      const double2* S0 = S_l(0);
      for_each_elem(n, [&](int i, int j, int idx) {
        const double2 s = sigmal[idx], st = cconj(sigmal[j + i * nn]);
        const double2 w = csub(s, st);
        if (ballistic) {
          gam[idx] = make_double2(-w.y, w.x);                         // Gamma_L = i (sL - sL^H)
        } else {
          double2 v = cscale(w, -fl);
          if (sl0) v = cadd(v, sl0[idx]);
          sig[idx] = v;
        }
        X[idx] = csub(zs_minus(z, S0, i, j, idx, H00[idx]), s);      // A = z S00 - H00 - sigmal
      });
      __syncthreads();
    }
    set_mixed(true);   // the device chain (mixed form)
    invert_X(Gl(0));
    const double2* GN1 = Gl(0);
    double2* GN1buf[2] = {tmp(T_GN1A), tmp(T_GN1B)};
    int gsel = 0;
    // sig<_L = -(sL - sL^H) fL = i fL Gamma_L with Gamma_L = L L^H, so every
    // left-connected g<_l = g^L_{l,1} sig<_L g^L_{l,1}^H is i fL V_l V_l^H
    // for the running column V_l = g^L_{l,1} L: one product per block.  An
    // indefinite Gamma_L has no such factor: sig<_L is formed and the
    // general recursion runs.
    const bool lowrank = ballistic && chol_psd(tmp(T_F3), tmp(T_SIG));
    if (ballistic && !lowrank) {
      for_each_elem(n, [&](int i, int j, int idx) {
        tmp(T_SIG)[idx] = cscale(csub(sigmal[idx], cconj(sigmal[j + i * nn])), -fl);
      });
      __syncthreads();
    }
    if (lowrank) {
      gemm_store(Gl(0), false, tmp(T_SIG), false, GN1buf[gsel]);   // V_1 = g_1 L
      GN1 = GN1buf[gsel];
      gsel ^= 1;
      gemm(GN1, false, GN1, true, [&](int i, int j, double2 v) {      // Gln(1) = i fL V V^H
        Gln(0)[i + j * nn] = make_double2(-v.y * fl, v.x * fl);
      });
    } else {
      gemm_store(Gl(0), false, tmp(T_SIG), false, tmp(T_F2));       // B = A sig
      gemm_store(tmp(T_F2), false, Gl(0), true, Gln(0));            // Gln(1) = B A^H
    }

    // ------------------------------------------------ forward sweep
    for (int l = 1; l <= nx - 2; l++) {
      const double2* H = blk(H1i, l);
      const double2* Hl = blk(Hii, l);
      const double2* srl = scat(sr, l, T_SRS);
      const double2* sll = scat(sl, l, T_SLS);
      const double2* Sl = S_l(l);
      gemm_store(H, false, Gl(l - 1), false, tmp(T_F1));            // B = H10 Gl(l-1)
      gemm(tmp(T_F1), false, H, true, [&](int i, int j, double2 v) { // A = z S - H00 - B H10^H
        const int idx = i + j * nn;
        const double2 h = srl ? cadd(Hl[idx], srl[idx]) : Hl[idx];
        X[idx] = csub(zs_minus(z, Sl, i, j, idx, h), v);
      });
      invert_X(Gl(l));
      if (want_T || lowrank) {  // g^L_{l,1} = g_l H_{l,l-1} g^L_{l-1,1} (low rank: times L)
        gemm_store(H, false, GN1, false, tmp(T_F1));
        gemm_store(Gl(l), false, tmp(T_F1), false, GN1buf[gsel]);
        GN1 = GN1buf[gsel];
        gsel ^= 1;
      }
      if (lowrank) {
        // Without scattering the recursion g<_l = g_l H g<_{l-1} H^H g_l^H
        // unrolls to g<_l = g^L_{l,1} sig<_L (g^L_{l,1})^H = i fL V_l V_l^H:
        // one product on the running column instead of four.
        gemm(GN1, false, GN1, true, [&](int i, int j, double2 v) {    // Gln(l) = i fL V V^H
          Gln(l)[i + j * nn] = make_double2(-v.y * fl, v.x * fl);
        });
      } else {
        gemm_store(H, false, Gln(l - 1), false, tmp(T_F2));         // B = H10 Gln(l-1)
        gemm(tmp(T_F2), false, H, true, [&](int i, int j, double2 v) { // C = B H10^H + sig<
          const int idx = i + j * nn;
          tmp(T_F3)[idx] = sll ? cadd(v, sll[idx]) : v;
        });
        gemm_store(Gl(l), false, tmp(T_F3), false, tmp(T_F4));      // B = A C
        gemm_store(tmp(T_F4), false, Gl(l), true, Gln(l));          // Gln(l) = B A^H
      }
    }

    // ------------------------------------------------ right contact, G_NN
    {
      const int l = nx - 1;
      const double2* Hl = blk(Hii, l);
      const double2* srl = scat(sr, l, T_SRS);
      for_each_elem(n, [&](int, int, int idx) {
        H00[idx] = srl ? cadd(Hl[idx], srl[idx]) : Hl[idx];
      });
      __syncthreads();
    }
    const double2* H = blk(H1i, nx - 1);
    set_mixed(false);  // the right lead in FP64
    const int itR = sancho(E, H00, H, false, tmp(T_GS), S_l(nx - 1));
    double2* sigmar = tmp(T_SIGR);
    gemm_store(H, true, tmp(T_GS), false, tmp(T_F1));               // A = H10^H G00
    gemm_store(tmp(T_F1), false, H, false, sigmar);                 // sigmar = A H10
    set_mixed(true);
    gemm_store(H, false, Gl(nx - 2), false, tmp(T_F2));             // B = H10 Gl(nx-1)
    {
      const double2* SN = S_l(nx - 1);
      gemm(tmp(T_F2), false, H, true, [&](int i, int j, double2 v) { // G00 = z S - H00 - sigmar - B H10^H
        const int idx = i + j * nn;
        X[idx] = csub(csub(zs_minus(z, SN, i, j, idx, H00[idx]), sigmar[idx]), v);
      });
    }
    double2* G00 = tmp(T_G00A);
    double2* G00n = tmp(T_G00B);
    double2* Gn = tmp(T_GNA);
    double2* Gnn = tmp(T_GNB);
    invert_X(G00, tk.ldos ? wblk(tk.ldos, nx - 1) : nullptr);
    const double fR = fermi((E - mur) / (o.boltz * templ));      // TEMPl: as the reference (:4051)
    gemm_store(H, false, Gln(nx - 2), false, tmp(T_F3));            // B = H10 Gln(nx-1)
    {
      const double2* sll = scat(sl, nx - 1, T_SLS);
      gemm(tmp(T_F3), false, H, true, [&](int i, int j, double2 v) { // sig = -(sR - sR^H) fR + C + sig<
        const int idx = i + j * nn;
        const double2 s = sigmar[idx], st = cconj(sigmar[j + i * nn]);
        double2 w = cadd(cscale(csub(s, st), -fR), v);
        if (sll) w = cadd(w, sll[idx]);
        tmp(T_SIG)[idx] = w;
      });
    }
    gemm_store(G00, false, tmp(T_SIG), false, tmp(T_F4));           // B = G00 sig
    {
      double2* nd = tk.ndens ? wblk(tk.ndens, nx - 1) : nullptr;
      double2* pd = tk.pdens ? wblk(tk.pdens, nx - 1) : nullptr;
      // the running G^> of green_RGF_CMS's recursion starts from this block's
      double2* gpn = (tk.GGi1 || (cms && tk.pdens)) ? tmp(T_GPN) : nullptr;
      gemm(tmp(T_F4), false, G00, true, [&](int i, int j, double2 v) {  // Gn = B G00^H
        const int idx = i + j * nn;
        Gn[idx] = v;
        if (nd) nd[idx] = v;
        if (pd || gpn) {
          const double2 gp = cadd(v, csub(G00[idx], cconj(G00[j + i * nn])));
          if (pd) pd[idx] = gp;
          if (gpn) gpn[idx] = gp;
        }
      });
    }
    {
      // tr = -Re sum_i [ (A1 Gp)_ii - (A2 Gn)_ii ],  A1 = -(sR - sR^H) fR, A2 = -(sR - sR^H)(fR - 1)
      double acc = 0.0;
      for_each_elem(n, [&](int i, int k, int idx) {
        const double2 gam = cscale(csub(sigmar[idx], cconj(sigmar[k + i * nn])), -1.0);
        const int ki = k + i * nn;
        const double2 gn = Gn[ki];
        const double2 gp = cadd(gn, csub(G00[ki], cconj(G00[idx])));
        const double2 b = cmul(cscale(gam, fR), gp);
        const double2 c = cmul(cscale(gam, fR - 1.0), gn);
        acc += b.x - c.x;
      });
      const double s = block_sum2(make_double2(acc, 0.0), sm.red).x;
      if (tk.tr && threadIdx.x == 0) *tk.tr = -s;
    }
    if (want_T) {
      gemm_store(H, false, GN1, false, tmp(T_X1));                  // H_{N,N-1} g^L_{N-1,1} (L)
      gemm_store(G00, false, tmp(T_X1), false, tmp(T_X2));          // G_{N1} (L)
      for_each_elem(n, [&](int i, int j, int idx) {                 // Gamma = i (Sigma - Sigma^H)
        const double2 dl = csub(sigmal[idx], cconj(sigmal[j + i * nn]));
        const double2 dr = csub(sigmar[idx], cconj(sigmar[j + i * nn]));
        tmp(T_GAML)[idx] = make_double2(-dl.y, dl.x);
        tmp(T_GAMR)[idx] = make_double2(-dr.y, dr.x);
      });
      __syncthreads();
      gemm_store(tmp(T_GAMR), false, tmp(T_X2), false, tmp(T_Y));   // Gamma_R G_N1 (L)
      if (lowrank) {
        // X2 = G_N1 L: T = Tr[Gamma_R X2 X2^H] = sum_ij Re (Gamma_R X2)_ij conj(X2_ij)
        double acc = 0.0;
        for_each_elem(n, [&](int, int, int idx) {
          const double2 y = tmp(T_Y)[idx], x = tmp(T_X2)[idx];
          acc += y.x * x.x + y.y * x.y;
        });
        const double tt = block_sum2(make_double2(acc, 0.0), sm.red).x;
        if (threadIdx.x == 0) *tk.T = tt;
      } else {
        gemm_store(tmp(T_GAML), false, tmp(T_X2), true, tmp(T_Z));  // Gamma_L G_N1^H
        const double2 tt = trace_prod(n, tmp(T_Y), tmp(T_Z), sm.red);
        if (threadIdx.x == 0) *tk.T = tt.x;
      }
    }

    // ------------------------------------------------ backward sweep
    // (skipped when no requested output depends on it: T and tr come from
    // the forward sweep and the right closure alone)
    const bool need_cur = tk.cur != nullptr;
    const bool need_q4 = need_cur || tk.GLi1 != nullptr;
    const bool need_back = tk.ldos || tk.ndens || tk.pdens || tk.GRi1 || tk.GLi1 || tk.GGi1 ||
                           tk.cur || tk.tre;
    // no scattering Sigma^<: every Gl< is anti-Hermitian by construction
    // (g Sigma^<_lead g^H and g H Gl< H^H g^H with anti-Hermitian factors)
    if (need_cur)
      for_each_elem(n, [&](int, int, int idx) { blk2(tk.cur, nx - 1)[idx] = 0.0; });
    if (need_back) publish(progress, 1);   // block nx-1: from the right closure
    for (int l = need_back ? nx - 2 : -1; l >= 0; l--) {
      const double2* Hb = blk(H1i, o.consistent ? l + 1 : l);
      const double2* gl = Gl(l);
      const double2* gln = Gln(l);
      double* curl = need_cur ? blk2(tk.cur, l) : nullptr;
      gemm_store(gl, false, Hb, true, tmp(T_Q1));                   // Gl H10^H
      if (need_cur) {
        gemm_store(Gn, false, tmp(T_Q1), true, tmp(T_P2));          // G<_{l+1} H10 Gl^H = G<_{l+1} Q1^H
        gemm_store(Hb, false, gln, false, tmp(T_P3));               // H10 Gl<
        gemm(G00, false, tmp(T_P3), false, [&](int i, int j, double2 v) {
          const int idx = i + j * nn;
          tmp(T_P4)[idx] = cadd(tmp(T_P2)[idx], v);                 // C + A
        });
        gemm(Hb, true, tmp(T_P4), false, [&](int i, int j, double2 v) {  // G<_{l+1,l}
          curl[i + j * nn] = v.x;
        });
      }
      gemm_store(tmp(T_Q1), false, Gn, false, tmp(T_Q2));           // Gl H10^H G<
      if (!ballistic || need_q4)
        gemm_store(gln, false, Hb, true, tmp(T_Q3));                // Gl< H10^H
      if (need_q4) {
        double2* gli = tk.GLi1 ? wblk(tk.GLi1, l) : nullptr;
        gemm(tmp(T_Q3), false, G00, true, [&](int i, int j, double2 v) {
          const int idx = i + j * nn;
          const double2 w = cadd(tmp(T_Q2)[idx], v);                // G<_{l,l+1}
          tmp(T_Q4)[idx] = w;
          if (gli) gli[idx] = w;
        });
        if (need_cur)
          gemm(Hb, false, tmp(T_Q4), false, [&](int i, int j, double2 v) {
            const int idx = i + j * nn;
            curl[idx] = curl[idx] - v.x;
          });
      }
      if (tk.GGi1) {  // the reference's GGi1: Gl^H H10^H Gp (+ Glp terms, which are zero); Gp
                      // is G^>_NN in green_RGF_RS, the running G^>_{l+1} in green_RGF_CMS
        gemm_store(gl, true, Hb, true, tmp(T_R1));
        gemm_store(tmp(T_R1), false, tmp(T_GPN), false, wblk(tk.GGi1, l));
      }
      double2* GN0 = tmp(T_F1);
      gemm_store(tmp(T_Q1), false, G00, false, GN0, tk.GRi1 ? wblk(tk.GRi1, l) : nullptr);  // G_{l,l+1}
      gemm_store(GN0, false, Hb, false, tmp(T_R5));                  // GN0 H10
      gemm(tmp(T_R5), false, gl, false, [&](int i, int j, double2 v) {
        const int idx = i + j * nn;
        G00n[idx] = cadd(gl[idx], v);                                 // G_ll = Gl + C
      });
      gemm(tmp(T_Q2), false, tmp(T_Q1), true, [&](int i, int j, double2 v) {
        const int idx = i + j * nn;
        Gnn[idx] = cadd(gln[idx], v);                               // Gn = Gl< + Gl H10^H G< H10 Gl^H
      });
      double2* T3 = tmp(T_X3);
      if (ballistic) {
        gemm_store(tmp(T_R5), false, gln, false, T3);                // GN0 H10 Gl<
      } else {
        gemm(tmp(T_R5), false, gln, false, [&](int i, int j, double2 v) {
          const int idx = i + j * nn;
          Gnn[idx] = cadd(Gnn[idx], v);                             // Gn += GN0 H10 Gl<
        });
        gemm(tmp(T_Q3), false, GN0, true, [&](int i, int j, double2 v) {
          const int idx = i + j * nn;
          Gnn[idx] = cadd(Gnn[idx], v);                             // Gn += Gl< H10^H GN0^H
        });
      }
      {
        // Ballistic: the last term Gl< H10^H GN0^H is -(GN0 H10 Gl<)^H, since
        // every Gl< is anti-Hermitian when no scattering Sigma^< enters.
        // The block outputs leave in one contiguous pass each (sequential
        // stores, which matters when they are host memory written through its
        // device mapping) rather than from the product epilogues.
        double2* ld = tk.ldos ? wblk(tk.ldos, l) : nullptr;
        double2* nd = tk.ndens ? wblk(tk.ndens, l) : nullptr;
        double2* pd = (tk.pdens && !cms) ? wblk(tk.pdens, l) : nullptr;
        if (ballistic || ld || nd || pd) {
          for_each_elem(n, [&](int i, int j, int idx) {
            const double2 g = G00n[idx];
            double2 w = Gnn[idx];
            if (ballistic) {
              w = cadd(w, csub(T3[idx], cconj(T3[j + i * nn])));
              Gnn[idx] = w;
            }
            if (ld) ld[idx] = g;
            if (nd) nd[idx] = w;
            if (pd) pd[idx] = cadd(w, csub(g, cconj(G00n[j + i * nn])));
          });
          __syncthreads();
        }
      }
      if (cms && (tk.pdens || tk.GGi1)) {
        // green_RGF_CMS's G^> (:4353-4369) with its never-filled Glp (zero):
        // Gp = Gl H10^H Gp H10 Gl^H
        double2* pd = tk.pdens ? wblk(tk.pdens, l) : nullptr;
        gemm_store(tmp(T_Q1), false, tmp(T_GPN), false, tmp(T_R1));
        gemm(tmp(T_R1), false, tmp(T_Q1), true, [&](int i, int j, double2 v) {
          const int idx = i + j * nn;
          tmp(T_GPN)[idx] = v;
          if (pd) pd[idx] = v;
        });
      }
      double2* t1 = G00; G00 = G00n; G00n = t1;
      double2* t2 = Gn; Gn = Gnn; Gnn = t2;
      publish(progress, nx - l);
    }

    // ------------------------------------------------ left trace (tre)
    if (tk.tre) {
      const double fl2 = fermi((E - mul) / (o.boltz * tempr));   // TEMPr: as the reference (:4152)
      double acc = 0.0;
      for_each_elem(n, [&](int i, int k, int idx) {
        const double2 gam = cscale(csub(sigmal[idx], cconj(sigmal[k + i * nn])), -1.0);
        const int ki = k + i * nn;
        const double2 gn = Gn[ki];
        const double2 gp = cadd(gn, csub(G00[ki], cconj(G00[idx])));
        const double2 b = cmul(cscale(gam, fl2), gp);
        const double2 c = cmul(cscale(gam, fl2 - 1.0), gn);
        acc += b.x - c.x;
      });
      const double s = block_sum2(make_double2(acc, 0.0), sm.red).x;
      if (threadIdx.x == 0) *tk.tre = s;
    }
    if (info && threadIdx.x == 0) {
      info->status = status;
      info->sancho_iters_left = itL;
      info->sancho_iters_right = itR;
      info->n_gemm = n_gemm;
      info->n_inv = n_inv;
    }
    __syncthreads();
  }


  // ------------------------------------------------------------------ adjoint
  // Stein doubling for X = Q + P X R with Q = -g g, P = g H^H, R = H g: the
  // energy derivative of a Sancho-Rubio surface Green's function g that
  // satisfies g = (z - H00 - H^H g H)^-1 (H = the coupling argument).
  // Result in out.  Uses temps T_F1..T_F4, T_Q1..T_Q3.
  // conj_h: the coupling argument is Hc^H (left lead).
  __device__ void dg_dE(const double2* g, const double2* Hc, bool conj_h, double2* out) {
    const int nn = n;
    double2 *P = tmp(T_Q1), *R = tmp(T_Q2), *P2 = tmp(T_Q3), *R2 = tmp(T_F4), *Y = tmp(T_F3);
    gemm_store(g, false, Hc, !conj_h, P);                            // P = g H^H
    gemm_store(Hc, conj_h, g, false, R);                             // R = H g
    gemm(g, false, g, false, [&](int i, int j, double2 v) { out[i + j * nn] = make_double2(-v.x, -v.y); });
    for (int it = 0; it < 4 * o.sancho_nmax; it++) {
      gemm_store(P, false, out, false, Y);                           // P X
      double dsum = 0.0, xsum = 0.0;
      gemm(Y, false, R, false, [&](int i, int j, double2 v) {        // X += P X R
        const int idx = i + j * nn;
        const double2 x = cadd(out[idx], v);
        out[idx] = x;
        dsum += fabs(v.x) + fabs(v.y);
        xsum += fabs(x.x) + fabs(x.y);
      });
      const double2 sums = block_sum2(make_double2(dsum, xsum), sm.red);
      if (!(sums.x > 1e-17 * sums.y)) break;
      gemm_store(P, false, P, false, P2);
      gemm_store(R, false, R, false, R2);
      double2* t1 = P; P = P2; P2 = t1;
      double2* t2 = R; R = R2; R2 = t2;
    }
  }

  // T(E), dT/dV_l (l = 0..nx-1) and dT/ds for one energy of a ballistic
  // device (no scattering self-energy).  V_l adds V_l * I to H_ll; the two
  // end blocks also shift their semi-infinite leads (the leads are the
  // continuation of Hii(:,:,1) / Hii(:,:,nx), as in green_RGF_RS), which
  // enters through dSigma/dE.  s scales the interior couplings H1i(:,:,m),
  // m = 2..nx-1 (1-based).  Reverse sweep with sqrt(nx) checkpoints of the
  // left-connected g_l and of the running column c_l = g^L_{l,1}.
  // green_rgf_calc_w (green_rgf.f90:3399-3831) == RGF_W (rgf_mod.f90:242-674)
  // with NBC = 0 and no off-diagonal P blocks (every call site).  V = the
  // device's (Vii, V1i); M = I - V P^R is formed block by block as needed:
  //   right-to-left  xlr_l = (M_ll - M_{l,l+1} xlr_{l+1} M_{l+1,l})^-1,
  //                  Wlr_l = xlr_l (V_ll - M_{l,l+1} xlr_{l+1} V_{l+1,l})   (:3710-3722)
  //   left-to-right  WR_l = Wlr_l - xlr_l M_{l,l-1} Wo_{l-1},
  //                  Wo_l = (V1i_l^T - WR_l M1i_l^T) xlr_{l+1}^T              (:3740-3778)
  //   W^< / W^>      WR P WR^H + Wi_j P Wi_j^T (-1) + Wi_m^T P Wi_m (-1)      (:3786-3829)
  // with Wi = i Im(Wo) (the routine zeroes the real part), j = l (l = nx-1:
  // nx-2), m = max(l-1, 0).  Plain transposes are materialised in epilogues
  // or one pass (the tensor-core GEMM takes N and C operands).  The
  // routine's LL / LG, wln / wlp and XR are never returned and are not
  // formed.  xlr lives in Gl(l), Wlr in Gln(l).
  __device__ void run_w(const DWTask& tk, const DDev& dv, DInfo* info) {
    const int nn = n;
    const double2* Vii = dv.Hii;
    const double2* V1i = dv.H1i;
    auto blk = [&](const double2* base, int l) { return base + (size_t)l * n2; };
    auto wblk = [&](double2* base, int l) { return base + (size_t)l * n2; };
    const double2* PR = tk.PR;
    // ---- right-to-left: xlr, Wlr
    {
      const int l = nx - 1;
      gemm(blk(Vii, l), false, blk(PR, l), false, [&](int i, int j, double2 v) {   // M_ll = I - V P^R
        X[i + j * nn] = (i == j) ? make_double2(1.0 - v.x, -v.y) : make_double2(-v.x, -v.y);
      });
      invert_X(Gl(l));
      gemm_store(Gl(l), false, blk(Vii, l), false, Gln(l));
    }
    for (int l = nx - 2; l >= 0; l--) {
      gemm(blk(V1i, l), true, blk(PR, l + 1), false, [&](int i, int j, double2 v) {
        tmp(T_F1)[i + j * nn] = make_double2(-v.x, -v.y);                         // M_{l,l+1}
      });
      gemm_store(tmp(T_F1), false, Gl(l + 1), false, tmp(T_F2));                  // B = M_{l,l+1} xlr_{l+1}
      gemm_store(tmp(T_F2), false, blk(V1i, l), false, tmp(T_F3));                // B V_{l+1,l}
      // X is only written by the epilogue of the last product before the
      // inverse: for nb <= 64 it shares shared memory with the GEMM staging
      gemm(blk(Vii, l), false, blk(PR, l), false, [&](int i, int j, double2 v) {   // M_ll
        tmp(T_SA)[i + j * nn] = (i == j) ? make_double2(1.0 - v.x, -v.y) : make_double2(-v.x, -v.y);
      });
      gemm(tmp(T_F3), false, blk(PR, l), false, [&](int i, int j, double2 v) {     // - B M_{l+1,l} = + B V P
        const int idx = i + j * nn;
        X[idx] = cadd(tmp(T_SA)[idx], v);
      });
      invert_X(Gl(l));
      for_each_elem(n, [&](int, int, int idx) { tmp(T_F4)[idx] = csub(blk(Vii, l)[idx], tmp(T_F3)[idx]); });
      __syncthreads();
      gemm_store(Gl(l), false, tmp(T_F4), false, Gln(l));                         // Wlr_l
    }
    // ---- left-to-right: WR, Wo; W^< and W^> block by block
    double2* WRc = tmp(T_G00A);
    double2 *M1c = tmp(T_H10A), *M1p = tmp(T_H10B), *M1T = tmp(T_H01A);
    double2 *Woc = tmp(T_GNA), *Wop = tmp(T_GNB);
    double2 *Wic = tmp(T_Q1), *NWTc = tmp(T_Q2), *Wip = tmp(T_Q3), *NWTp = tmp(T_Q4);
    double2* xT = tmp(T_R5);
    for (int l = 0; l < nx; l++) {
      double2* wr_out = wblk(tk.WR, l);
      if (l == 0) {
        for_each_elem(n, [&](int, int, int idx) {
          const double2 w = Gln(0)[idx];
          WRc[idx] = w;
          wr_out[idx] = w;
        });
        __syncthreads();
      } else {
        gemm_store(Gl(l), false, M1p, false, tmp(T_F1));                          // xlr_l M_{l,l-1}
        gemm(tmp(T_F1), false, Wop, false, [&](int i, int j, double2 v) {
          const int idx = i + j * nn;
          const double2 w = csub(Gln(l)[idx], v);
          WRc[idx] = w;
          wr_out[idx] = w;
        });
      }
      if (l < nx - 1) {
        gemm(blk(V1i, l), false, blk(PR, l), false, [&](int i, int j, double2 v) {  // M_{l+1,l} and its transpose
          const double2 m = make_double2(-v.x, -v.y);
          M1c[i + j * nn] = m;
          M1T[j + i * nn] = m;
        });
        for_each_elem(n, [&](int i, int j, int idx) { xT[j + i * nn] = Gl(l + 1)[idx]; });
        __syncthreads();
        gemm(WRc, false, M1T, false, [&](int i, int j, double2 v) {               // C = V1i^T - WR M1i^T
          const int idx = i + j * nn;
          tmp(T_F2)[idx] = csub(blk(V1i, l)[j + i * nn], v);
        });
        double2* wo_out = tk.WRi1 ? wblk(tk.WRi1, l) : nullptr;
        gemm(tmp(T_F2), false, xT, false, [&](int i, int j, double2 v) {          // Wo_l = C xlr_{l+1}^T
          const int idx = i + j * nn;
          Woc[idx] = v;
          if (wo_out) wo_out[idx] = v;
          const double2 wi = make_double2(0.0 * v.x, v.y);                        // real part zeroed
          Wic[idx] = wi;
          NWTc[j + i * nn] = make_double2(-wi.x, -wi.y);                          // -(Wi)^T
        });
      }
      // W^< / W^> of block l (the off-diagonal terms use Wi_j, Wi_m)
      const double2 *Wj, *NWTj, *Wm, *NWTm;
      const int jp = l < nx - 1 ? l + 1 : l;
      if (l < nx - 1) { Wj = Wic; NWTj = NWTc; } else { Wj = Wip; NWTj = NWTp; }
      if (l == 0) { Wm = Wic; NWTm = NWTc; } else { Wm = Wip; NWTm = NWTp; }
      for (int which = 0; which < 2; which++) {
        const double2* P = which == 0 ? tk.PL : tk.PG;
        double2* out = wblk(which == 0 ? tk.WL : tk.WG, l);
        gemm_store(WRc, false, blk(P, l), false, tmp(T_F1));                      // WR P
        gemm_store(tmp(T_F1), false, WRc, true, out);                             // WR P WR^H
        gemm_store(Wj, false, blk(P, jp), false, tmp(T_F1));                      // Wi_j P_j'
        gemm(tmp(T_F1), false, NWTj, false, [&](int i, int j, double2 v) {
          const int idx = i + j * nn;
          out[idx] = cadd(out[idx], v);
        });
        gemm_store(NWTm, false, blk(P, (l > 0 ? l - 1 : 0)), false, tmp(T_F1));   // -Wi_m^T P_m
        gemm(tmp(T_F1), false, Wm, false, [&](int i, int j, double2 v) {
          const int idx = i + j * nn;
          out[idx] = cadd(out[idx], v);
        });
      }
      double2* t;
      t = M1c; M1c = M1p; M1p = t;
      t = Woc; Woc = Wop; Wop = t;
      t = Wic; Wic = Wip; Wip = t;
      t = NWTc; NWTc = NWTp; NWTp = t;
    }
    if (info && threadIdx.x == 0) {
      info->status = status;
      info->sancho_iters_left = 0;
      info->sancho_iters_right = 0;
      info->n_gemm = n_gemm;
      info->n_inv = n_inv;
    }
    __syncthreads();
  }

  __device__ void run_adjoint(const DAdj& tk, const DDev& dv, DInfo* info) {
    const int nn = n;
    const double E = tk.E;
    const double2 z = make_double2(E, o.eta_dev);
    const double2* Hii = dv.Hii;
    const double2* H1i = dv.H1i;
    auto blk = [&](const double2* base, int l) { return base + (size_t)l * n2; };
    const int nl = nx - 1;                     // blocks of the left-connected chain: 0..nx-2
    int S = nl;                                // segment length
    if (nl > 16) { S = 1; while (S * S < nl) S++; }
    const int nseg = (nl + S - 1) / S;
    // storage in the Gl / Gln regions: [checkpoints (nseg) | segment (S)]
    const int cko = nseg > 1 ? nseg : 0;
    auto ckg = [&](int q) { return Gl(q); };
    auto ckc = [&](int q) { return Gln(q); };
    auto sgg = [&](int q) { return Gl(cko + q); };
    auto sgc = [&](int q) { return Gln(cko + q); };
    double2* H00 = tmp(T_H00);
    // ---- left lead
    for_each_elem(n, [&](int, int, int idx) { H00[idx] = Hii[idx]; });
    __syncthreads();
    const int itL = sancho(E, H00, blk(H1i, 0), true, tmp(T_GS));
    double2* sigmal = tmp(T_SIGL);
    gemm_store(blk(H1i, 0), false, tmp(T_GS), false, tmp(T_F1));
    gemm_store(tmp(T_F1), false, blk(H1i, 0), true, sigmal);
    double2* dSL = tmp(T_Q4);                                        // -dSigma_L/dE
    dg_dE(tmp(T_GS), blk(H1i, 0), true, tmp(T_F2));                 // coupling argument H1i(1)^H
    gemm_store(blk(H1i, 0), false, tmp(T_F2), false, tmp(T_F1));
    gemm(tmp(T_F1), false, blk(H1i, 0), true, [&](int i, int j, double2 v) {
      dSL[i + j * nn] = make_double2(-v.x, -v.y);
    });
    // ---- forward sweep with checkpoints
    double2* gprev = tmp(T_GN1A);  // rolling g_{l-1}, c_{l-1} when checkpointing
    double2* cprev = tmp(T_GN1B);
    auto store_state = [&](int l, const double2* g, const double2* c) {
      if (nseg == 1) {
        if (g != sgg(l)) for_each_elem(n, [&](int, int, int idx) { sgg(l)[idx] = g[idx]; sgc(l)[idx] = c[idx]; });
        else for_each_elem(n, [&](int, int, int idx) { sgc(l)[idx] = c[idx]; });
        __syncthreads();
      } else if (l % S == 0) {
        for_each_elem(n, [&](int, int, int idx) { ckg(l / S)[idx] = g[idx]; ckc(l / S)[idx] = c[idx]; });
        __syncthreads();
      }
    };
    // g_0
    for_each_elem(n, [&](int i, int j, int idx) {
      const double2 h = Hii[idx];
      const double2 a = (i == j) ? make_double2(z.x - h.x, z.y - h.y) : make_double2(-h.x, -h.y);
      X[idx] = csub(a, sigmal[idx]);
    });
    __syncthreads();
    double2* g0 = nseg == 1 ? sgg(0) : gprev;
    invert_X(g0);
    store_state(0, g0, g0);
    if (nseg > 1) for_each_elem(n, [&](int, int, int idx) { cprev[idx] = g0[idx]; });
    __syncthreads();
    const double2* gl = g0;
    const double2* cl = nseg == 1 ? sgc(0) : cprev;
    // forward step from (g_{l-1}, c_{l-1}) to (g_l, c_l) into (gout, cout)
    auto fwd_step = [&](int l, const double2* gp, const double2* cp, double2* gout, double2* cout) {
      const double2* Hc = blk(H1i, l);
      const double2* Hl = blk(Hii, l);
      gemm_store(Hc, false, gp, false, tmp(T_F1));
      gemm(tmp(T_F1), false, Hc, true, [&](int i, int j, double2 v) {
        const int idx = i + j * nn;
        const double2 h = Hl[idx];
        const double2 a = (i == j) ? make_double2(z.x - h.x, z.y - h.y) : make_double2(-h.x, -h.y);
        X[idx] = csub(a, v);
      });
      invert_X(gout);
      gemm_store(Hc, false, cp, false, tmp(T_F1));
      gemm_store(gout, false, tmp(T_F1), false, cout);               // c_l = g_l H_{l,l-1} c_{l-1}
    };
    for (int l = 1; l <= nx - 2; l++) {
      if (nseg == 1) {
        fwd_step(l, sgg(l - 1), sgc(l - 1), sgg(l), sgc(l));
        gl = sgg(l);
        cl = sgc(l);
      } else {
        double2* gn = tmp(T_G00A);
        double2* cn = tmp(T_G00B);
        fwd_step(l, gprev, cprev, gn, cn);
        store_state(l, gn, cn);
        for_each_elem(n, [&](int, int, int idx) { gprev[idx] = gn[idx]; cprev[idx] = cn[idx]; });
        __syncthreads();
        gl = gprev;
        cl = cprev;
      }
    }
    // ---- right lead, G_NN, X = G_{N1}, T, W
    const double2* Hr = blk(H1i, nx - 1);
    for_each_elem(n, [&](int, int, int idx) { H00[idx] = blk(Hii, nx - 1)[idx]; });
    __syncthreads();
    const int itR = sancho(E, H00, Hr, false, tmp(T_GS));
    double2* sigmar = tmp(T_SIGR);
    gemm_store(Hr, true, tmp(T_GS), false, tmp(T_F1));
    gemm_store(tmp(T_F1), false, Hr, false, sigmar);
    double2* dSR = tmp(T_R5);                                        // -dSigma_R/dE
    dg_dE(tmp(T_GS), Hr, false, tmp(T_F2));
    gemm_store(Hr, true, tmp(T_F2), false, tmp(T_F1));
    gemm(tmp(T_F1), false, Hr, false, [&](int i, int j, double2 v) { dSR[i + j * nn] = make_double2(-v.x, -v.y); });
    gemm_store(Hr, false, gl, false, tmp(T_F1));
    gemm(tmp(T_F1), false, Hr, true, [&](int i, int j, double2 v) {
      const int idx = i + j * nn;
      const double2 h = H00[idx];
      double2 a = (i == j) ? make_double2(z.x - h.x, z.y - h.y) : make_double2(-h.x, -h.y);
      a = csub(a, sigmar[idx]);
      X[idx] = csub(a, v);
    });
    double2* GNN = tmp(T_G00A);  // gn of the checkpointed forward loop is dead here
    invert_X(GNN);
    double2* XN1 = tmp(T_X2);
    gemm_store(Hr, false, cl, false, tmp(T_F1));
    gemm_store(GNN, false, tmp(T_F1), false, XN1);                    // X = G_NN H c_{N-2}
    double2* gamL = tmp(T_GAML);
    double2* gamR = tmp(T_GAMR);
    double2* dgL = tmp(T_H10B);
    double2* dgR = tmp(T_H01A);
    for_each_elem(n, [&](int i, int j, int idx) {
      const double2 dl = csub(sigmal[idx], cconj(sigmal[j + i * nn]));
      const double2 dr = csub(sigmar[idx], cconj(sigmar[j + i * nn]));
      gamL[idx] = make_double2(-dl.y, dl.x);
      gamR[idx] = make_double2(-dr.y, dr.x);
      const double2 el = csub(dSL[idx], cconj(dSL[j + i * nn]));     // i (S' - S'^H)
      const double2 er = csub(dSR[idx], cconj(dSR[j + i * nn]));
      dgL[idx] = make_double2(-el.y, el.x);
      dgR[idx] = make_double2(-er.y, er.x);
    });
    __syncthreads();
    double2* W = tmp(T_SIG);
    gemm_store(gamL, false, XN1, true, tmp(T_F1));                    // Gamma_L X^H
    gemm_store(tmp(T_F1), false, gamR, false, W);                     // W = Gamma_L X^H Gamma_R
    double2* XGX = tmp(T_F3);
    gemm_store(gamR, false, XN1, false, tmp(T_F1));                   // Gamma_R X
    gemm_store(XN1, false, gamL, false, tmp(T_F2));                   // X Gamma_L
    gemm_store(tmp(T_F2), false, XN1, true, XGX);                     // X Gamma_L X^H
    const double T = trace_prod(n, gamR, XGX, sm.red).x;
    // lead terms: Tr[Gamma_R X dGamma_L X^H] and Tr[dGamma_R X Gamma_L X^H]
    gemm_store(tmp(T_F1), false, dgL, false, tmp(T_F2));              // Gamma_R X dGamma_L
    gemm_store(tmp(T_F2), false, XN1, true, tmp(T_F4));
    double leadL = 0.0, leadR = 0.0;
    {
      double acc = 0.0;
      for (int i = threadIdx.x; i < n; i += kThreads) acc += tmp(T_F4)[i + i * nn].x;
      leadL = block_sum2(make_double2(acc, 0.0), sm.red).x;
    }
    leadR = trace_prod(n, dgR, XGX, sm.red).x;
    // ---- reverse sweep
    double2 *r1 = tmp(T_Q1), *r0 = tmp(T_Q2), *k1 = tmp(T_Q3), *k0 = tmp(T_GNA);
    double2 *y1 = tmp(T_H01B), *y0 = tmp(T_HSS), *tA = tmp(T_F1), *tB = tmp(T_F2);
    // l = nx-1: r = G_NN, k = X
    for_each_elem(n, [&](int, int, int idx) { r1[idx] = GNN[idx]; k1[idx] = XN1[idx]; });
    __syncthreads();
    gemm_store(W, false, r1, false, y1);                              // Y = W r
    double gN = 2.0 * trace_prod(n, k1, y1, sm.red).x;
    // right lead term 2 Re Tr[W r_{N-1} S'_R X]
    gemm_store(y1, false, dSR, false, tA);
    gN += 2.0 * trace_prod(n, tA, XN1, sm.red).x + leadR;
    if (threadIdx.x == 0) tk.dTdV[nx - 1] = gN;
    double ds = 0.0;
    for (int sg = nseg - 1; sg >= 0; sg--) {
      const int l0 = sg * S, l1 = (l0 + S < nl) ? l0 + S : nl;
      if (nseg > 1) {  // recompute the segment from its checkpoint
        for_each_elem(n, [&](int, int, int idx) { sgg(0)[idx] = ckg(sg)[idx]; sgc(0)[idx] = ckc(sg)[idx]; });
        __syncthreads();
        for (int l = l0 + 1; l < l1; l++) fwd_step(l, sgg(l - 1 - l0), sgc(l - 1 - l0), sgg(l - l0), sgc(l - l0));
      }
      for (int l = l1 - 1; l >= l0; l--) {
        const double2* g = sgg(l - l0);
        const double2* c = sgc(l - l0);
        const double2* Hn = blk(H1i, l + 1);                          // H_{l+1,l}
        gemm_store(r1, false, Hn, false, tA);
        gemm_store(tA, false, g, false, r0);                          // r_l = r_{l+1} H_{l+1,l} g_l
        gemm_store(g, false, Hn, true, tA);
        gemm(tA, false, k1, false, [&](int i, int j, double2 v) {     // k_l = c_l + g_l H^H k_{l+1}
          const int idx = i + j * nn;
          k0[idx] = cadd(c[idx], v);
        });
        gemm_store(W, false, r0, false, y0);                          // Y_l = W r_l
        double gl_ = 2.0 * trace_prod(n, k0, y0, sm.red).x;
        if (l == 0) {  // left lead: 2 Re Tr[W X S'_L k_0] + Tr[Gamma_R X dGamma_L X^H]
          gemm_store(W, false, XN1, false, tA);
          gemm_store(tA, false, dSL, false, tB);
          gl_ += 2.0 * trace_prod(n, tB, k0, sm.red).x + leadL;
        }
        if (threadIdx.x == 0) tk.dTdV[l] = gl_;
        const int m = l + 1;                                          // coupling H_{m,m-1}
        if (m >= 1 && m <= nx - 2) {
          gemm_store(y1, false, Hn, false, tA);                       // Y_m H_{m,m-1}
          double t1 = trace_prod(n, tA, k0, sm.red).x;
          gemm_store(y0, false, Hn, true, tB);                        // Y_{m-1} H^H
          t1 += trace_prod(n, tB, k1, sm.red).x;
          ds += 2.0 * t1;
        }
        double2* t;
        t = r1; r1 = r0; r0 = t;
        t = k1; k1 = k0; k0 = t;
        t = y1; y1 = y0; y0 = t;
      }
    }
    if (threadIdx.x == 0) {
      if (tk.T) *tk.T = T;
      if (tk.dTds) *tk.dTds = ds;
    }
    if (info && threadIdx.x == 0) {
      info->status = status;
      info->sancho_iters_left = itL;
      info->sancho_iters_right = itR;
      info->n_gemm = n_gemm;
      info->n_inv = n_inv;
    }
    __syncthreads();
  }

  __device__ double* blk2(double* base, int l) const { return base + (size_t)l * n2; }
};

// One task (drop-in solve or adjoint) with policy Ops.  The slot holds
// Gl[nx], Gln[nx] and the scratch blocks of this task's own nx and nb.
template <class Ops>
__device__ __forceinline__ void solve_task(const KParams& p, int64_t t, double2* slot, Smem& sm,
                                           double2* dyn_smem) {
  DInfo* info = p.info ? p.info + t : nullptr;
  const int dev = p.adj ? p.adj[t].dev : (p.wtasks ? p.wtasks[t].dev : p.tasks[t].dev);
  const DDev dv = p.devs[dev];
  const int n = (int)dv.nm;
  const size_t n2 = (size_t)n * n;
  double2* temps = slot + 2 * (size_t)dv.nx * n2;
  Ops ops(sm.inv, dyn_smem, temps + (size_t)T_INV * n2, temps + (size_t)T_RT * n2, n);
  Solver<Ops> s(p.o, dv.nx, sm, ops, slot, n, (int)dv.nx);
  if (p.adj) s.run_adjoint(p.adj[t], dv, info);
  else if (p.wtasks) s.run_w(p.wtasks[t], dv, info);
  else s.run(p.tasks[t], dv, info, p.progress ? p.progress + t : nullptr);
}

}  // namespace

}  // namespace rgf
