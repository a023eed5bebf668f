// slvfe.cu -- slvfe's free-energy functional (chmpot) for one data set on the GPU, in FP64,
// with slvfe's default options (sfemain.F90:22-64): py-hnc, regularised Cholesky solve of
// the reference-solvent equation, eczr zero shift, harmonic extrapolation weights, linear
// extrapolation of omega in solution, normalize 'yes', no bin merging.
//
//   k_slv_prep     distnorm's per-species scaling of rho / rho0 (slvfe.F90:1467-1502) and
//                  omega in solution where both distributions are sampled (getslncv :875-930)
//   k_slv_distnorm the chi0 row scaling (slvfe.F90:1503-1525): Gauss-Seidel sweeps over the
//                  bins in one CTA, each bin's correction from the corrections already
//                  updated in this sweep, to 1e-8 within 100 sweeps
//   k_slv_extrap   omega in solution for bins sampled on one side only (:930-1001): a
//                  weighted linear fit over the species' sampled bins, a thread per bin
//   k_slv_reg      the per-species regularisation trace / count^2 (getinscv :1003-1120)
//   k_slv_build    A = chi0 - rho0 rho0^T (+ reg per species block, 1 on unsampled
//                  diagonals), padded to a multiple of the tile with the identity
//   k_chol_*       blocked right-looking Cholesky of A (32 x 32 FP64 tiles: diagonal
//                  factor, panel solve, trailing update)
//   k_slv_solve    forward and backward substitution for the reference-solvent omega
//   k_slv_check    posv_wrap's acceptance of that solution (slvfe.F90:520-531): the
//                  largest residual against the regularised matrix, the largest element
//   eigen-decomposition fallback (getinscv :1124-1170), when the Cholesky factor fails
//   or the check rejects the solution: the unregularised matrix (k_slv_unreg) goes to
//   cuSOLVER's Dsyevd, as the reference's syevr_wrap sends it to cusolverDnSsyevd; its
//   first nsp eigenpairs are skipped in the pseudo-inverse (k_slv_evd_coef, k_slv_evd_x)
//   k_slv_chmpot   the eczr zero shift, the functional and its per-species sums (:744-803)
//
// Every reduction is a fixed-order tree, so a run is reproducible bit for bit.
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <cmath>
#include <cstdint>
#include <vector>

#include "../../include/ermod_slvfe.h"

namespace {

constexpr int kTile = 32;
constexpr int kNT = 1024;          // threads of the single-CTA kernels
constexpr int kMaxSpecies = 16;
constexpr double kTol = 1.0e-8;    // distnorm convergence (slvfe.F90:1520)
constexpr int kItrMax = 100;
constexpr double kTiny = 1.0e-8;   // zero-bin tie (slvfe.F90:1180)

enum : int { kOk = 0, kErrNorm = 1, kErrExtrap = 2, kErrChol = 3, kErrZero = 4 };

thread_local const char* g_err = "";

// the first failing step's code stays: later kernels run on, as the host learns of it only at the end
__device__ void set_status(int* st, int code) { atomicCAS(st, 0, code); }

__device__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// fixed-order sum of one value per thread of a kNT-thread block
__device__ double block_sum(double v, double* sh) {
  v = warp_sum(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  if (w == 0) {
    double r = l < kNT / 32 ? sh[l] : 0.0;
    r = warp_sum(r);
    if (l == 0) sh[0] = r;
  }
  __syncthreads();
  return sh[0];
}

__device__ double block_max(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  if (w == 0) {
    double r = l < kNT / 32 ? sh[l] : -INFINITY;
    for (int o = 16; o > 0; o >>= 1) r = fmax(r, __shfl_down_sync(0xffffffffu, r, o));
    if (l == 0) sh[0] = r;
  }
  __syncthreads();
  return sh[0];
}

__device__ double block_min(double v, double* sh) { return -block_max(-v, sh); }

struct SlvArgs {
  int n, nsp;
  double kT;
  int n0;               // bins as read (before grouping)
  const double* rd0;    // rho in solution as read, for getslncv's threshold (slvfe.F90:884)
  const double* rr0;    // rho0 as read
  const double* rd;     // rho in solution as read (engstore-normalised)
  const double* rr;     // rho0 in the reference solvent as read
  const double* crd;    // bin coordinates (engsln's bin_middle)
  const int* spec;      // 1-based species of each bin
  double* rho;          // scaled rho
  double* rho0;         // scaled rho0
  double* nummol;       // [nsp] molecules per species
  double* omega;        // omega in solution
  int* both;            // 1: sampled in both systems
  double* harm;         // rho rho0 / (rho + rho0)
  double* reg;          // [nsp]
  int* status;
  int functional;       // ERMOD_SLVFE_PYHNC / HNC / THNC / NONE
  double et;            // thnc threshold (kcal/mol)
};

// ---- distnorm's scaling and the directly sampled omega -------------------------------
__global__ void __launch_bounds__(kNT) k_slv_prep(SlvArgs a) {
  __shared__ double sh[32];
  const int n = a.n;
  for (int p = 1; p <= a.nsp; ++p) {
    double s = 0.0, s0 = 0.0;
    for (int i = threadIdx.x; i < n; i += kNT)
      if (a.spec[i] == p) { s += a.rd[i]; s0 += a.rr[i]; }
    s = block_sum(s, sh);
    s0 = block_sum(s0, sh);
    const double nm = rint(s);
    if (threadIdx.x == 0) a.nummol[p - 1] = nm;
    const double f = s > 0.0 ? nm / s : 0.0, f0 = s0 > 0.0 ? nm / s0 : 0.0;
    for (int i = threadIdx.x; i < n; i += kNT)
      if (a.spec[i] == p) { a.rho[i] = a.rd[i] * f; a.rho0[i] = a.rr[i] * f0; }
  }
  __syncthreads();
  double mn = INFINITY, mn0 = INFINITY;
  for (int i = threadIdx.x; i < a.n0; i += kNT) {
    if (a.rd0[i] > 0.0) mn = fmin(mn, a.rd0[i]);
    if (a.rr0[i] > 0.0) mn0 = fmin(mn0, a.rr0[i]);
  }
  mn = block_min(mn, sh);
  mn0 = block_min(mn0, sh);
  for (int i = threadIdx.x; i < n; i += kNT) {
    const double r = a.rho[i], r0 = a.rho0[i];
    const double rs = fmin(r / mn, 10.0), rr = fmin(r0 / mn0, 10.0);
    const int b = (rint(rs) >= 1.0 && rint(rr) >= 1.0) ? 1 : 0;
    a.both[i] = b;
    a.omega[i] = b ? -a.kT * log(r / r0) - a.crd[i] : 0.0;
    const double hs = r + r0;
    a.harm[i] = hs > 0.0 ? r * r0 / hs : 0.0;
  }
}

// ---- chmpot's grouping of consecutive bins (slvfe.F90:609-698) ------------------------
// merged bin k covers the bins [rng[k].x, rng[k].y) as read; rng[k].z = 1 for the last merged
// bin of a species, whose coordinate is that species' last coordinate as read
__global__ void k_slv_merge_vec(int g, const int4* __restrict__ rng, const double* __restrict__ rd,
                                const double* __restrict__ rr, const double* __restrict__ crd,
                                const int* __restrict__ spec, double* __restrict__ mrd, double* __restrict__ mrr,
                                double* __restrict__ mcrd, int* __restrict__ mspec) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= g) return;
  const int4 r = rng[k];
  double s = 0.0, s0 = 0.0, c = 0.0;
  for (int i = r.x; i < r.y; ++i) { s += rd[i]; s0 += rr[i]; c += crd[i]; }
  mrd[k] = s;
  mrr[k] = s0;
  mcrd[k] = r.z ? crd[r.y - 1] : c / (double)(r.y - r.x);
  mspec[k] = spec[r.x];
}

// column-major g x g sums of the n0 x n0 matrix over the bins of each merged pair, fixed order
__global__ void k_slv_merge_mat(int g, int n0, const int4* __restrict__ rng, const double* __restrict__ chi0,
                                double* __restrict__ chi) {
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (size_t)g * g) return;
  const int r = (int)(e % g), c = (int)(e / g);
  const int4 R = rng[r], Cc = rng[c];
  double s = 0.0;
  for (int j = Cc.x; j < Cc.y; ++j)
    for (int i = R.x; i < R.y; ++i) s += chi0[(size_t)j * n0 + i];
  chi[e] = s;
}

// ---- chi0 row scaling: Gauss-Seidel sweeps in one CTA --------------------------------
__global__ void __launch_bounds__(kNT) k_slv_distnorm(SlvArgs a, double* __restrict__ chi) {
  extern __shared__ double corr[];            // [n]
  __shared__ double part[32 * kMaxSpecies];
  __shared__ double sh[32];
  const int n = a.n, nsp = a.nsp;
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  for (int i = threadIdx.x; i < n; i += kNT) corr[i] = 1.0;
  __syncthreads();
  for (int it = 0;; ++it) {
    for (int i = 0; i < n; ++i) {
      const double* col = chi + (size_t)i * n;
      double acc[kMaxSpecies];
      for (int p = 0; p < nsp; ++p) acc[p] = 0.0;
      for (int j = threadIdx.x; j < n; j += kNT) {
        const double v = corr[j] * col[j];
        const int p = a.spec[j] - 1;
        for (int q = 0; q < nsp; ++q) acc[q] += q == p ? v : 0.0;
      }
      for (int p = 0; p < nsp; ++p) {
        const double v = warp_sum(acc[p]);
        if (l == 0) part[w * kMaxSpecies + p] = v;
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        double s = 0.0;
        for (int p = 0; p < nsp; ++p) {
          double d = 0.0;
          for (int q = 0; q < kNT / 32; ++q) d += part[q * kMaxSpecies + p];
          if (d > 0.0) s += a.nummol[p] / d;
        }
        corr[i] = s / nsp * a.rho0[i];
      }
      __syncthreads();
    }
    // chi *= corr corr^T
    for (size_t e = threadIdx.x; e < (size_t)n * n; e += kNT) {
      const int r = (int)(e % n), c = (int)(e / n);
      chi[e] *= corr[r] * corr[c];
    }
    double err = 0.0;
    for (int i = threadIdx.x; i < n; i += kNT)
      if (a.rho0[i] > 0.0) err = fmax(err, fabs(corr[i] - 1.0));
    err = block_max(err, sh);
    if (err <= kTol) return;
    if (it + 1 >= kItrMax) {
      if (threadIdx.x == 0) set_status(a.status, kErrNorm);
      return;
    }
  }
}

// ---- omega in solution where one distribution is empty: weighted linear fit ----------
__global__ void k_slv_extrap(SlvArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = a.n;
  if (i >= n || a.both[i]) return;
  if (a.rho[i] <= 0.0) { a.omega[i] = 0.0; return; }
  const int sp = a.spec[i];
  auto same = [&](int k) { return a.spec[k] == sp && a.both[k]; };
  int m = 0, k = n - 1;
  for (int q = i - 1; q >= 0; --q) if (same(q)) { m = q; break; }
  for (int q = i + 1; q < n; ++q) if (same(q)) { k = q; break; }
  int j;
  if (a.both[m] && a.both[k]) j = abs(m - i) < abs(k - i) ? m : k;
  else if (a.both[m] || a.both[k]) j = a.both[m] ? m : k;
  else { set_status(a.status, kErrExtrap); return; }
  const double kT = a.kT, cj = a.crd[j], ci = a.crd[i];
  double wsum = 0.0;
  for (int q = 0; q < n; ++q) {
    if (!same(q)) continue;
    double sh = a.crd[q] - cj;
    if (q < i) sh = -sh - 2.0 * (cj - ci);
    const double wq = exp(-sh / kT) * a.harm[q];
    if (wq > 0.0) wsum += wq;
  }
  double m1 = 0.0, m2 = 0.0, my = 0.0, mxy = 0.0;
  for (int q = 0; q < n; ++q) {
    if (!same(q)) continue;
    double sh = a.crd[q] - cj;
    if (q < i) sh = -sh - 2.0 * (cj - ci);
    double wq = exp(-sh / kT) * a.harm[q];
    if (!(wq > 0.0)) continue;
    wq /= wsum;
    const double x = a.crd[q], y = a.omega[q];
    m1 += wq * x; m2 += wq * x * x; my += wq * y; mxy += wq * x * y;
  }
  const double den = m2 - m1 * m1;
  const double c0 = (m2 * my - m1 * mxy) / den, c1 = (mxy - m1 * my) / den;
  a.omega[i] = c0 + c1 * ci;
}

// ---- regularisation per species: trace of the sampled block / count^2 ----------------
__global__ void __launch_bounds__(kNT) k_slv_reg(SlvArgs a, const double* __restrict__ chi) {
  __shared__ double sh[32];
  const int n = a.n;
  for (int p = 1; p <= a.nsp; ++p) {
    double t = 0.0, c = 0.0;
    for (int i = threadIdx.x; i < n; i += kNT)
      if (a.spec[i] == p && a.rho0[i] > 0.0) {
        t += chi[(size_t)i * n + i] - a.rho0[i] * a.rho0[i];
        c += 1.0;
      }
    t = block_sum(t, sh);
    c = block_sum(c, sh);
    if (threadIdx.x == 0) a.reg[p - 1] = c > 0.0 ? t / (c * c) : 0.0;
  }
}

// ---- the padded system matrix and right-hand side ------------------------------------
__global__ void k_slv_build(SlvArgs a, const double* __restrict__ chi, int N, double* __restrict__ A,
                            double* __restrict__ b) {
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (size_t)N * N) return;
  const int r = (int)(e % N), c = (int)(e / N);   // column-major
  const int n = a.n;
  double v;
  if (r >= n || c >= n) {
    v = r == c ? 1.0 : 0.0;
  } else {
    const bool pr = a.rho0[r] > 0.0, pc = a.rho0[c] > 0.0;
    if (pr && pc) {
      v = chi[(size_t)c * n + r] - a.rho0[r] * a.rho0[c];
      if (a.spec[r] == a.spec[c]) v += a.reg[a.spec[r] - 1];
    } else {
      v = r == c ? 1.0 : 0.0;
    }
  }
  A[e] = v;
  if (c == 0) b[r] = (r < n && a.rho0[r] > 0.0) ? -a.kT * (a.rho[r] - a.rho0[r]) : 0.0;
}

// ---- blocked Cholesky, lower, column-major, 32 x 32 tiles ----------------------------
__global__ void __launch_bounds__(kTile * kTile) k_chol_diag(double* __restrict__ A, int N, int kt, int* status) {
  __shared__ double t[kTile][kTile + 1];
  const int r = threadIdx.x % kTile, c = threadIdx.x / kTile, k0 = kt * kTile;
  t[r][c] = A[(size_t)(k0 + c) * N + k0 + r];
  __syncthreads();
  for (int j = 0; j < kTile; ++j) {
    if (r == j && c == j) {
      const double d = t[j][j];
      if (!(d > 0.0)) set_status(status, kErrChol);
      t[j][j] = sqrt(fmax(d, 1e-300));
    }
    __syncthreads();
    if (c == j && r > j) t[r][j] /= t[j][j];
    __syncthreads();
    if (c > j && r >= c) t[r][c] -= t[r][j] * t[c][j];
    __syncthreads();
  }
  if (r >= c) A[(size_t)(k0 + c) * N + k0 + r] = t[r][c];
}

// tiles below the diagonal: X L_kk^T = A_ik, a thread per row of the tile
__global__ void __launch_bounds__(kTile) k_chol_panel(double* __restrict__ A, int N, int kt) {
  __shared__ double L[kTile][kTile + 1];
  const int r = threadIdx.x, k0 = kt * kTile, i0 = (kt + 1 + blockIdx.x) * kTile;
  for (int c = 0; c < kTile; ++c) L[r][c] = A[(size_t)(k0 + c) * N + k0 + r];
  __syncthreads();
  double x[kTile];
  for (int c = 0; c < kTile; ++c) x[c] = A[(size_t)(k0 + c) * N + i0 + r];
  for (int c = 0; c < kTile; ++c) {
    double v = x[c];
    for (int l = 0; l < c; ++l) v -= x[l] * L[c][l];
    x[c] = v / L[c][c];
  }
  for (int c = 0; c < kTile; ++c) A[(size_t)(k0 + c) * N + i0 + r] = x[c];
}

// trailing update A_ij -= A_ik A_jk^T for the lower tiles i >= j > k
__global__ void __launch_bounds__(kTile * kTile) k_chol_update(double* __restrict__ A, int N, int kt) {
  __shared__ double P[kTile][kTile + 1], Q[kTile][kTile + 1];
  // blockIdx.x enumerates the lower-triangle tile pairs (i, j), j <= i, of the trailing matrix
  int b = blockIdx.x, j = 0;
  const int m = N / kTile - kt - 1;
  while (b >= m - j) { b -= m - j; ++j; }
  const int i = j + b;
  const int r = threadIdx.x % kTile, c = threadIdx.x / kTile;
  const int k0 = kt * kTile, i0 = (kt + 1 + i) * kTile, j0 = (kt + 1 + j) * kTile;
  P[r][c] = A[(size_t)(k0 + c) * N + i0 + r];
  Q[r][c] = A[(size_t)(k0 + c) * N + j0 + r];
  __syncthreads();
  double s = 0.0;
  for (int l = 0; l < kTile; ++l) s += P[r][l] * Q[c][l];
  A[(size_t)(j0 + c) * N + i0 + r] -= s;
}

// ---- L L^T x = b, one CTA: tiles of forward then backward substitution ---------------
__global__ void __launch_bounds__(kNT) k_slv_solve(const double* __restrict__ A, int N, double* __restrict__ b) {
  __shared__ double xs[kTile];
  const int nt = N / kTile;
  for (int kt = 0; kt < nt; ++kt) {      // L y = b
    const int k0 = kt * kTile;
    if (threadIdx.x == 0)
      for (int c = 0; c < kTile; ++c) {
        double v = b[k0 + c];
        for (int l = 0; l < c; ++l) v -= A[(size_t)(k0 + l) * N + k0 + c] * xs[l];
        xs[c] = v / A[(size_t)(k0 + c) * N + k0 + c];
        b[k0 + c] = xs[c];
      }
    __syncthreads();
    for (int r = k0 + kTile + threadIdx.x; r < N; r += kNT) {
      double v = 0.0;
      for (int l = 0; l < kTile; ++l) v += A[(size_t)(k0 + l) * N + r] * xs[l];
      b[r] -= v;
    }
    __syncthreads();
  }
  for (int kt = nt - 1; kt >= 0; --kt) { // L^T x = y
    const int k0 = kt * kTile;
    if (threadIdx.x == 0)
      for (int c = kTile - 1; c >= 0; --c) {
        double v = b[k0 + c];
        for (int l = c + 1; l < kTile; ++l) v -= A[(size_t)(k0 + c) * N + k0 + l] * xs[l];
        xs[c] = v / A[(size_t)(k0 + c) * N + k0 + c];
        b[k0 + c] = xs[c];
      }
    __syncthreads();
    for (int r = threadIdx.x; r < k0; r += kNT) {   // row r of L^T is column r of L
      double v = 0.0;
      for (int l = 0; l < kTile; ++l) v += A[(size_t)r * N + k0 + l] * xs[l];
      b[r] -= v;
    }
    __syncthreads();
  }
}

// ---- posv_wrap's acceptance (slvfe.F90:520-531) against the regularised matrix Areg ----
constexpr double kPosvResidual = 1.0e-6, kPosvAbs = 1.0e6;

__global__ void __launch_bounds__(kNT) k_slv_check(int n, int N, const double* __restrict__ Areg,
                                                   const double* __restrict__ rhs, const double* __restrict__ x,
                                                   double* __restrict__ out) {
  __shared__ double sh[32];
  double res = 0.0, big = 0.0;
  for (int r = threadIdx.x; r < n; r += kNT) {
    double v = 0.0;
    for (int c = 0; c < n; ++c) v += Areg[(size_t)c * N + r] * x[c];
    res = fmax(res, fabs(v - rhs[r]));
    big = fmax(big, fabs(x[r]));
  }
  res = block_max(res, sh);
  big = block_max(big, sh);
  if (threadIdx.x == 0) { out[0] = res; out[1] = big; }
}

// ---- the eigen-decomposition fallback (getinscv, slvfe.F90:1124-1170) ------------------
// E = chi0 - rho0 rho0^T on the sampled bins, the identity elsewhere (n x n, column-major)
__global__ void k_slv_unreg(SlvArgs a, const double* __restrict__ chi, double* __restrict__ E) {
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int n = a.n;
  if (e >= (size_t)n * n) return;
  const int r = (int)(e % n), c = (int)(e / n);
  const bool pr = a.rho0[r] > 0.0, pc = a.rho0[c] > 0.0;
  E[e] = (pr && pc) ? chi[(size_t)c * n + r] - a.rho0[r] * a.rho0[c] : (r == c ? 1.0 : 0.0);
}

// coef[i] = (sum over sampled bins p of -kT (rho - rho0)_p V[p][i]) / lambda_i for i >= nsp
__global__ void k_slv_evd_coef(SlvArgs a, const double* __restrict__ V, const double* __restrict__ lam,
                               double* __restrict__ coef) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = a.n;
  if (i >= n) return;
  double s = 0.0;
  if (i >= a.nsp) {
    for (int p = 0; p < n; ++p)
      if (a.rho0[p] > 0.0) s += -a.kT * (a.rho[p] - a.rho0[p]) * V[(size_t)i * n + p];
    s /= lam[i];
  }
  coef[i] = s;
}

// x[p] = sum over i >= nsp of V[p][i] coef[i]
__global__ void k_slv_evd_x(SlvArgs a, const double* __restrict__ V, const double* __restrict__ coef,
                            double* __restrict__ x) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = a.n;
  if (p >= n) return;
  double s = 0.0;
  for (int i = a.nsp; i < n; ++i) s += V[(size_t)i * n + p] * coef[i];
  x[p] = s;
}

__device__ double pyhnc_soln(double f) { return f < 0.0 ? f + f / (exp(-f) - 1.0) + 1.0 : f / 2.0; }
__device__ double pyhnc_refs(double f) { return f < 0.0 ? log1p(-f) * (1.0 / f - 1.0) + 1.0 : f / 2.0; }

// chmpot's integrands (slvfe.F90:759-774): py-hnc, hnc / thnc (thnc, :1417-1436), none
__device__ void functional_terms(int functional, double om, double om0, double kT, double et, double* ls,
                                 double* lr) {
  switch (functional) {
    case ERMOD_SLVFE_HNC: *ls = om / kT / 2.0; *lr = om0 / kT / 2.0; return;
    case ERMOD_SLVFE_THNC: *ls = om / kT / 2.0; *lr = om0 < et ? 0.0 : om0 / kT / 2.0; return;
    case ERMOD_SLVFE_NONE: *ls = 0.0; *lr = 0.0; return;
    default: *ls = pyhnc_soln(om / kT); *lr = pyhnc_refs(om0 / kT); return;
  }
}

// ---- eczr zero shift, the functional and its per-species sums ------------------------
__global__ void __launch_bounds__(kNT) k_slv_chmpot(SlvArgs a, const double* __restrict__ x,
                                                    const double* __restrict__ aveuv, double* __restrict__ chmpt) {
  __shared__ double sh[32];
  __shared__ double zx[kMaxSpecies];
  const int n = a.n;
  if (threadIdx.x < a.nsp) {   // the last bin pair of the species around zero energy
    const int p = threadIdx.x + 1;
    int k = -1, prev = -1;
    for (int q = 0; q < n; ++q) {
      if (a.spec[q] != p) continue;
      if (prev >= 0 && q == prev + 1 && a.crd[prev] <= 0.0 && 0.0 <= a.crd[q]) {
        const double lo = fabs(a.crd[prev]), hi = a.crd[q];
        if (hi > lo + kTiny) k = prev;
        else if (hi < lo - kTiny) k = q;
        else k = a.rho0[prev] >= a.rho0[q] ? prev : q;
      }
      prev = q;
    }
    if (k < 0) set_status(a.status, kErrZero);
    zx[threadIdx.x] = k >= 0 ? x[k] : 0.0;
  }
  __syncthreads();
  const double kT = a.kT;
  for (int p = 1; p <= a.nsp; ++p) {
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += kNT) {
      if (a.spec[i] != p) continue;
      const double r = a.rho[i], r0 = a.rho0[i];
      if (!(r > 0.0 || r0 > 0.0)) continue;
      const double om0 = (r0 > 0.0 ? -kT * (r - r0) / r0 - x[i] : 0.0) + zx[p - 1];
      const double hs = r + r0;
      const double wt = r >= r0 ? 1.0 : 1.0 - ((r - r0) / (hs > 0.0 ? hs : 1.0)) * ((r - r0) / (hs > 0.0 ? hs : 1.0));
      double ls, lr;
      functional_terms(a.functional, a.omega[i], om0, kT, a.et, &ls, &lr);
      const double fac = wt * ls + (1.0 - wt) * lr;
      const double lcent = -(a.omega[i] + a.crd[i]);
      s += -kT * (r - r0) + lcent * r + kT * fac * (r - r0);
    }
    s = block_sum(s, sh);
    if (threadIdx.x == 0) chmpt[p - 1] = s + aveuv[p - 1];
  }
}

int fail(int code, const char* name) {
  g_err = name;
  return code;
}

template <class T>
cudaError_t dalloc(T** p, size_t n) { return cudaMalloc((void**)p, sizeof(T) * (n ? n : 1)); }

}  // namespace

extern "C" const char* ermod_slvfe_last_error(void) { return g_err; }

extern "C" int32_t ermod_slvfe_delta_mu(int32_t device, int32_t n0, int32_t nsp, int32_t group, int32_t inft,
                                        const double* rho_sln, const double* rho_ref, const double* chi_ref,
                                        const double* crd, const int32_t* spec, double kT, const double* aveuv,
                                        double slfeng, double* chmpt, double* total) {
  const ermod_slvfe_opts o{ERMOD_SLVFE_PYHNC, 1, 0.0};
  return ermod_slvfe_delta_mu_ex(device, n0, nsp, group, inft, rho_sln, rho_ref, chi_ref, crd, spec, kT, aveuv,
                                 slfeng, &o, chmpt, total, nullptr);
}

extern "C" int32_t ermod_slvfe_delta_mu_ex(int32_t device, int32_t n0, int32_t nsp, int32_t group, int32_t inft,
                                           const double* rho_sln, const double* rho_ref, const double* chi_ref,
                                           const double* crd, const int32_t* spec, double kT, const double* aveuv,
                                           double slfeng, const ermod_slvfe_opts* opts, double* chmpt,
                                           double* total, int32_t* used_evd) {
  if (used_evd) *used_evd = 0;
  if (n0 < 2 || nsp < 1 || nsp > kMaxSpecies || group < 1 || inft < 0 || inft > 100 || !rho_sln || !rho_ref || !chi_ref || !crd || !spec ||
      !aveuv || !chmpt || !(kT > 0.0) || !opts || opts->functional < ERMOD_SLVFE_PYHNC ||
      opts->functional > ERMOD_SLVFE_NONE)
    return fail(ERMOD_ERR_ARG, "slv_arg");
  for (int i = 0; i < n0; ++i)
    if (spec[i] < 1 || spec[i] > nsp || (i > 0 && spec[i] < spec[i - 1])) return fail(ERMOD_ERR_ARG, "slv_arg");
  // chmpot's grouping (slvfe.F90:613-640): per species (bins - rduvcore * inft / 100) / group
  // merged bins, the last one taking the rest; rduvcore, the bins since the coordinate spacing
  // last stayed constant, counted as datread does (slvfe.F90:114-135).  The index bookkeeping
  // is host work, the sums run on the device.
  std::vector<int4> rng;
  for (int i = 0; i < n0;) {
    int j = i;
    while (j < n0 && spec[j] == spec[i]) ++j;
    int core = 0;
    double dprev = 0.0;
    for (int q = i + 1; q < j; ++q) {
      const double d = crd[q] - crd[q - 1];
      if (q - i + 1 > 2) core = std::fabs(d - dprev) < 1.0e-8 ? 0 : core + 1;
      dprev = d;
    }
    const int m = (j - i - core * inft / 100) / group;
    if (m < 1) return fail(ERMOD_ERR_ARG, "slv_grp");
    for (int q = 0; q < m; ++q)
      rng.push_back(make_int4(i + q * group, q < m - 1 ? i + (q + 1) * group : j, q == m - 1 ? 1 : 0, 0));
    i = j;
  }
  const int n = (int)rng.size();
  if (n < 2) return fail(ERMOD_ERR_ARG, "slv_grp");
  if ((size_t)n * sizeof(double) > 160 * 1024) return fail(ERMOD_ERR_ARG, "slv_siz");   // corr in shared memory
  if (cudaSetDevice(device) != cudaSuccess) return fail(ERMOD_ERR_CUDA, "slv_cud");
  const int N = (n + kTile - 1) / kTile * kTile;
  const size_t nn = (size_t)n * n, NN = (size_t)N * N, nn0 = (size_t)n0 * n0;
  double *d_rd0 = nullptr, *d_rr0 = nullptr, *d_crd0 = nullptr, *d_chi0 = nullptr;
  double *d_rd = nullptr, *d_rr = nullptr, *d_crd = nullptr, *d_chi = nullptr, *d_rho = nullptr, *d_rho0 = nullptr;
  double *d_nm = nullptr, *d_om = nullptr, *d_harm = nullptr, *d_reg = nullptr, *d_A = nullptr, *d_b = nullptr;
  double *d_av = nullptr, *d_out = nullptr, *d_A2 = nullptr, *d_rhs = nullptr, *d_chk = nullptr;
  double *d_E = nullptr, *d_lam = nullptr, *d_coef = nullptr, *d_work = nullptr;
  int *d_spec0 = nullptr, *d_spec = nullptr, *d_both = nullptr, *d_st = nullptr, *d_info = nullptr;
  int4* d_rng = nullptr;
  cudaStream_t st = nullptr;
  cusolverDnHandle_t sol = nullptr;
  int rc = ERMOD_OK;
  auto cleanup = [&]() {
    for (void* p : {(void*)d_rd0, (void*)d_rr0, (void*)d_crd0, (void*)d_chi0, (void*)d_rd, (void*)d_rr,
                    (void*)d_crd, (void*)d_chi, (void*)d_rho, (void*)d_rho0, (void*)d_nm, (void*)d_om,
                    (void*)d_harm, (void*)d_reg, (void*)d_A, (void*)d_b, (void*)d_av, (void*)d_out,
                    (void*)d_spec0, (void*)d_spec, (void*)d_both, (void*)d_st, (void*)d_rng, (void*)d_A2,
                    (void*)d_rhs, (void*)d_chk, (void*)d_E, (void*)d_lam, (void*)d_coef, (void*)d_work,
                    (void*)d_info})
      if (p) cudaFree(p);
    if (sol) cusolverDnDestroy(sol);
    if (st) cudaStreamDestroy(st);
  };
  bool ok = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) == cudaSuccess;
  ok = ok && dalloc(&d_rd0, n0) == cudaSuccess && dalloc(&d_rr0, n0) == cudaSuccess;
  ok = ok && dalloc(&d_crd0, n0) == cudaSuccess && dalloc(&d_chi0, nn0) == cudaSuccess;
  ok = ok && dalloc(&d_spec0, n0) == cudaSuccess && dalloc(&d_rng, n) == cudaSuccess;
  ok = ok && dalloc(&d_rd, n) == cudaSuccess && dalloc(&d_rr, n) == cudaSuccess && dalloc(&d_crd, n) == cudaSuccess;
  ok = ok && dalloc(&d_chi, nn) == cudaSuccess && dalloc(&d_rho, n) == cudaSuccess && dalloc(&d_rho0, n) == cudaSuccess;
  ok = ok && dalloc(&d_nm, nsp) == cudaSuccess && dalloc(&d_om, n) == cudaSuccess && dalloc(&d_harm, n) == cudaSuccess;
  ok = ok && dalloc(&d_reg, nsp) == cudaSuccess && dalloc(&d_A, NN) == cudaSuccess && dalloc(&d_b, N) == cudaSuccess;
  ok = ok && dalloc(&d_av, nsp) == cudaSuccess && dalloc(&d_out, nsp) == cudaSuccess;
  ok = ok && dalloc(&d_spec, n) == cudaSuccess && dalloc(&d_both, n) == cudaSuccess && dalloc(&d_st, 1) == cudaSuccess;
  ok = ok && dalloc(&d_A2, NN) == cudaSuccess && dalloc(&d_rhs, N) == cudaSuccess && dalloc(&d_chk, 2) == cudaSuccess;
  if (!ok) { cleanup(); return fail(ERMOD_ERR_CUDA, "slv_mem"); }
  ok = cudaMemcpyAsync(d_rd0, rho_sln, 8 * n0, cudaMemcpyHostToDevice, st) == cudaSuccess;
  ok = ok && cudaMemcpyAsync(d_rr0, rho_ref, 8 * n0, cudaMemcpyHostToDevice, st) == cudaSuccess;
  ok = ok && cudaMemcpyAsync(d_crd0, crd, 8 * n0, cudaMemcpyHostToDevice, st) == cudaSuccess;
  ok = ok && cudaMemcpyAsync(d_chi0, chi_ref, 8 * nn0, cudaMemcpyHostToDevice, st) == cudaSuccess;
  ok = ok && cudaMemcpyAsync(d_spec0, spec, 4 * n0, cudaMemcpyHostToDevice, st) == cudaSuccess;
  ok = ok && cudaMemcpyAsync(d_rng, rng.data(), sizeof(int4) * n, cudaMemcpyHostToDevice, st) == cudaSuccess;
  ok = ok && cudaMemcpyAsync(d_av, aveuv, 8 * nsp, cudaMemcpyHostToDevice, st) == cudaSuccess;
  ok = ok && cudaMemsetAsync(d_st, 0, sizeof(int), st) == cudaSuccess;
  SlvArgs a{n, nsp, kT, n0, d_rd0, d_rr0, d_rd, d_rr, d_crd, d_spec, d_rho, d_rho0, d_nm, d_om, d_both, d_harm,
            d_reg, d_st, opts->functional, opts->et};
  const size_t corr_smem = (size_t)n * sizeof(double);
  if (ok && corr_smem > 48 * 1024)
    ok = cudaFuncSetAttribute(k_slv_distnorm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)corr_smem) ==
         cudaSuccess;
  if (ok) {
    k_slv_merge_vec<<<(n + 127) / 128, 128, 0, st>>>(n, d_rng, d_rd0, d_rr0, d_crd0, d_spec0, d_rd, d_rr, d_crd,
                                                     d_spec);
    k_slv_merge_mat<<<(unsigned)((nn + 255) / 256), 256, 0, st>>>(n, n0, d_rng, d_chi0, d_chi);
    k_slv_prep<<<1, kNT, 0, st>>>(a);
    k_slv_distnorm<<<1, kNT, corr_smem, st>>>(a, d_chi);
    k_slv_extrap<<<(n + 127) / 128, 128, 0, st>>>(a);
    k_slv_reg<<<1, kNT, 0, st>>>(a, d_chi);
    k_slv_build<<<(unsigned)((NN + 255) / 256), 256, 0, st>>>(a, d_chi, N, d_A, d_b);
    ok = cudaMemcpyAsync(d_A2, d_A, sizeof(double) * NN, cudaMemcpyDeviceToDevice, st) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(d_rhs, d_b, sizeof(double) * N, cudaMemcpyDeviceToDevice, st) == cudaSuccess;
    const int nt = N / kTile;
    for (int kt = 0; kt < nt; ++kt) {
      k_chol_diag<<<1, kTile * kTile, 0, st>>>(d_A, N, kt, d_st);
      const int m = nt - kt - 1;
      if (m > 0) {
        k_chol_panel<<<m, kTile, 0, st>>>(d_A, N, kt);
        k_chol_update<<<m * (m + 1) / 2, kTile * kTile, 0, st>>>(d_A, N, kt);
      }
    }
    k_slv_solve<<<1, kNT, 0, st>>>(d_A, N, d_b);
    k_slv_check<<<1, kNT, 0, st>>>(n, N, d_A2, d_rhs, d_b, d_chk);
    ok = ok && cudaGetLastError() == cudaSuccess;
  }
  // posv_wrap's verdict decides between the Cholesky solution and the eigen-decomposition
  int status = 0;
  double chk[2] = {0.0, 0.0};
  ok = ok && cudaMemcpyAsync(&status, d_st, sizeof(int), cudaMemcpyDeviceToHost, st) == cudaSuccess;
  ok = ok && cudaMemcpyAsync(chk, d_chk, sizeof(chk), cudaMemcpyDeviceToHost, st) == cudaSuccess;
  ok = ok && cudaStreamSynchronize(st) == cudaSuccess;
  const bool rejected = status == kErrChol || (status == kOk && !(chk[0] <= kPosvResidual && chk[1] <= kPosvAbs));
  if (ok && rejected && opts->evd) {
    int lwork = 0, info = 0;
    ok = dalloc(&d_E, nn) == cudaSuccess && dalloc(&d_lam, n) == cudaSuccess && dalloc(&d_coef, n) == cudaSuccess &&
         dalloc(&d_info, 1) == cudaSuccess;
    ok = ok && cusolverDnCreate(&sol) == CUSOLVER_STATUS_SUCCESS && cusolverDnSetStream(sol, st) == CUSOLVER_STATUS_SUCCESS;
    if (ok) {
      k_slv_unreg<<<(unsigned)((nn + 255) / 256), 256, 0, st>>>(a, d_chi, d_E);
      ok = cudaGetLastError() == cudaSuccess;
    }
    ok = ok && cusolverDnDsyevd_bufferSize(sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, n, d_E, n, d_lam,
                                           &lwork) == CUSOLVER_STATUS_SUCCESS;
    ok = ok && dalloc(&d_work, (size_t)lwork) == cudaSuccess;
    ok = ok && cusolverDnDsyevd(sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, n, d_E, n, d_lam, d_work, lwork,
                                d_info) == CUSOLVER_STATUS_SUCCESS;
    ok = ok && cudaMemcpyAsync(&info, d_info, sizeof(int), cudaMemcpyDeviceToHost, st) == cudaSuccess;
    ok = ok && cudaStreamSynchronize(st) == cudaSuccess;
    if (ok && info != 0) status = kErrChol;   // "Failed inversion of correlation matrix" (slvfe.F90:1134)
    if (ok && info == 0) {
      k_slv_evd_coef<<<(n + 127) / 128, 128, 0, st>>>(a, d_E, d_lam, d_coef);
      k_slv_evd_x<<<(n + 127) / 128, 128, 0, st>>>(a, d_E, d_coef, d_b);
      ok = cudaGetLastError() == cudaSuccess;
      if (status == kErrChol) {
        status = kOk;
        ok = ok && cudaMemsetAsync(d_st, 0, sizeof(int), st) == cudaSuccess;
      }
      if (used_evd) *used_evd = 1;
    }
  } else if (ok && rejected && status == kOk) {
    status = kErrChol;   // the solution posv_wrap rejects, with the fallback switched off
  }
  if (ok && status == kOk) {
    k_slv_chmpot<<<1, kNT, 0, st>>>(a, d_b, d_av, d_out);
    ok = cudaGetLastError() == cudaSuccess;
  }
  int status2 = 0;
  ok = ok && cudaMemcpyAsync(&status2, d_st, sizeof(int), cudaMemcpyDeviceToHost, st) == cudaSuccess;
  ok = ok && cudaMemcpyAsync(chmpt, d_out, 8 * nsp, cudaMemcpyDeviceToHost, st) == cudaSuccess;
  ok = ok && cudaStreamSynchronize(st) == cudaSuccess;
  if (status == kOk) status = status2;
  if (!ok) rc = fail(ERMOD_ERR_CUDA, "slv_cud");
  else if (status == kErrNorm) rc = fail(ERMOD_ERR_SLVFE, "slv_nrm");
  else if (status == kErrExtrap) rc = fail(ERMOD_ERR_SLVFE, "slv_ext");
  else if (status == kErrChol) rc = fail(ERMOD_ERR_SLVFE, "slv_chl");
  else if (status == kErrZero) rc = fail(ERMOD_ERR_SLVFE, "slv_zer");
  if (rc == ERMOD_OK && total) {
    double s = slfeng;
    for (int p = 0; p < nsp; ++p) s += chmpt[p];
    *total = s;
  }
  cleanup();
  return rc;
}
